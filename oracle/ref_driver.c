/*
 * ref_driver.c -- a flat C driver over the UNMODIFIED gviz reference, built
 * from the reference's own source files by oracle/Makefile into
 * oracle/_ref/libgviz_ref.so.
 *
 * TEST AND BASELINE INFRASTRUCTURE ONLY. It lets tests/ and the CPU legs of
 * bench.py run the reference's real gvizForceEmbedderStep
 * (src/embedders/gvizForceEmbedder.c:445-495) and real gvizQuadtree
 * (src/ds/gvizQuadtree.c) on inputs shared with libgvizcuda. It only calls
 * the reference's public API; no reference code is reproduced here.
 */
#include "ds/gvizGraph.h"
#include "ds/gvizQuadtree.h"
#include "ds/gvizSubgraph.h"
#include "embedders/gvizEmbeddedGraph.h"
#include "embedders/gvizForceEmbedder.h"
#include "utils/graphLoader.h"
#include "utils/graphs.h"

#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

/* same layout as orcParams (oracle/gviz_oracle.h) */
typedef struct refParams {
  int32_t model;
  int32_t barnesHutEnabled;
  int32_t preventOverlap;
  int32_t _pad;
  uint64_t nodesPerCell;
  double edgeLength;
  double theta;
  double gravityK;
  double radiusBase;
  double radiusPerDegree;
  double overlapConstant;
  double jitterTolerance;
} refParams;

typedef struct refLayout {
  gvizGraph g;
  gvizForceEmbedderState s;
  int initRes;
} refLayout;

static refLayout *finish_create(refLayout *r, int model) {
  gvizGraphBuildLayout(&r->g);
  gvizSubgraph sg = gvizSubgraphCreateFull(&r->g);
  r->initRes = gvizForceEmbedderInit(&r->s, sg, 2, (gvizForceModelKind)model);
  return r;
}

/* Graph from an ordered undirected edge list (gvizGraphAddEdge order). */
refLayout *ref_create_edges(size_t V, const uint32_t *ea, const uint32_t *eb,
                            size_t E, int model) {
  refLayout *r = calloc(1, sizeof(refLayout));
  if (!r)
    return NULL;
  gvizGraphInitAtCapacity(&r->g, 0, V ? V : 1);
  for (size_t i = 0; i < V; i++)
    gvizGraphAddVertex(&r->g, NULL, NULL, NULL);
  for (size_t e = 0; e < E; e++)
    gvizGraphAddEdge(&r->g, ea[e], eb[e]);
  return finish_create(r, model);
}

/* kind 0: build_rect_mesh(a, b); kind 1: build_random_connected_graph(a,
 * density, seed) (src/utils/graphs.c:285-316, 598-639). */
refLayout *ref_create_builtin(int kind, size_t a, size_t b, double density,
                              unsigned seed, int model) {
  refLayout *r = calloc(1, sizeof(refLayout));
  if (!r)
    return NULL;
  if (kind == 0)
    r->g = build_rect_mesh(a, b);
  else
    r->g = build_random_connected_graph(a, density, seed);
  return finish_create(r, model);
}

int ref_init_result(refLayout *r) { return r->initRes; }

/* The embedder state, for glue that attaches to it (gvizForceEmbedderState *). */
void *ref_state(refLayout *r) { return &r->s; }

int ref_invoke_toggle_overlap(refLayout *r) {
  return gvizEmbeddedGraphInvokeAction((gvizEmbeddedGraph *)&r->s,
                                       "forceEmbedder.toggleOverlapPrevention", NULL);
}
size_t ref_vertex_count(refLayout *r) { return r->s.vertexCount; }

void ref_configure(refLayout *r, const refParams *p, double boxExtent) {
  gvizForceEmbedderState *s = &r->s;
  gvizForceEmbedderConfigure(s, p->edgeLength, boxExtent);
  gvizForceEmbedderConfigureSpeed(s, p->jitterTolerance);
  gvizForceEmbedderConfigureBarnesHut(s, p->theta, (size_t)p->nodesPerCell);
  gvizForceEmbedderSetBarnesHutEnabled(s, p->barnesHutEnabled);
  gvizForceEmbedderConfigureGravity(s, p->gravityK);
  gvizForceEmbedderConfigureRadius(s, p->radiusBase, p->radiusPerDegree);
  gvizForceEmbedderConfigureOverlapPrevention(s, p->overlapConstant);
  gvizForceEmbedderSetPreventOverlapEnabled(s, p->preventOverlap);
}

/* Live toggles that the reference reads every step. */
void ref_set_prevent_overlap(refLayout *r, int on) {
  gvizForceEmbedderSetPreventOverlapEnabled(&r->s, on);
}
void ref_set_barnes_hut(refLayout *r, int on) {
  gvizForceEmbedderSetBarnesHutEnabled(&r->s, on);
}

int ref_begin(refLayout *r, unsigned seed) {
  return gvizForceEmbedderBegin(&r->s, seed);
}

double ref_box_extent(refLayout *r) { return r->s.boxExtent; }

/* CSR in compact order, read through the subgraph neighbour iterator
 * (src/ds/gvizSubgraph.c:466-519). Pass cols == NULL to get rowOff only. */
void ref_get_csr(refLayout *r, uint64_t *rowOff, uint32_t *cols) {
  gvizForceEmbedderState *s = &r->s;
  gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)s;
  size_t n = gvizGraphSize(eg->subgraph.g);
  size_t *compact = malloc(sizeof(size_t) * (n ? n : 1));
  for (size_t i = 0; i < n; i++)
    compact[i] = (size_t)-1;
  for (size_t i = 0; i < s->vertexCount; i++)
    compact[s->vertices[i]] = i;
  uint64_t off = 0;
  for (size_t i = 0; i < s->vertexCount; i++) {
    rowOff[i] = off;
    gvizSubgraphNeighborIterator it =
        gvizSubgraphNeighborIteratorCreate(&eg->subgraph, s->vertices[i]);
    size_t u;
    while (gvizSubgraphNeighborIterate(&it, &u)) {
      if (cols)
        cols[off] = (uint32_t)compact[u];
      off++;
    }
  }
  rowOff[s->vertexCount] = off;
  free(compact);
}

void ref_get_degree_mass(refLayout *r, uint64_t *degree, double *mass) {
  for (size_t i = 0; i < r->s.vertexCount; i++) {
    if (degree)
      degree[i] = r->s.degree[i];
    if (mass)
      mass[i] = r->s.mass[i];
  }
}

void ref_get_positions(refLayout *r, double *xy) {
  gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)&r->s;
  for (size_t i = 0; i < r->s.vertexCount; i++) {
    double *p = gvizEmbeddedGraphGetVPosition(eg, r->s.vertices[i]);
    xy[2 * i] = p[0];
    xy[2 * i + 1] = p[1];
  }
}

void ref_set_positions(refLayout *r, const double *xy) {
  gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)&r->s;
  for (size_t i = 0; i < r->s.vertexCount; i++) {
    double p[2] = {xy[2 * i], xy[2 * i + 1]};
    gvizEmbeddedGraphSetVPosition(eg, r->s.vertices[i], p);
  }
}

/* Overwrites the FA2 history so one step can be teacher-forced from a given
 * state: structForce becomes oldStructForce at the start of the next Step. */
void ref_set_fa2_state(refLayout *r, const double *structForce, double speed,
                       double efficiency) {
  if (structForce)
    memcpy(r->s.structForce, structForce, sizeof(double) * 2 * r->s.vertexCount);
  r->s.globalSpeed = speed;
  r->s.speedEfficiency = efficiency;
}

double ref_step(refLayout *r) { return gvizForceEmbedderStep(&r->s); }

int ref_run(refLayout *r, size_t maxIters, double eps) {
  return gvizForceEmbedderRun(&r->s, maxIters, eps);
}

int ref_invoke_step_action(refLayout *r) {
  return gvizEmbeddedGraphInvokeAction((gvizEmbeddedGraph *)&r->s,
                                       "forceEmbedder.step", NULL);
}

void ref_get_state(refLayout *r, double *disp, double *structForce,
                   double *att, double *rep, double *swing, double *traction,
                   double *applied, double *scalars) {
  gvizForceEmbedderState *s = &r->s;
  size_t V = s->vertexCount;
  if (disp)
    memcpy(disp, s->disp, sizeof(double) * 2 * V);
  if (structForce)
    memcpy(structForce, s->structForce, sizeof(double) * 2 * V);
  if (att)
    memcpy(att, s->attForceMag, sizeof(double) * V);
  if (rep)
    memcpy(rep, s->repForceMag, sizeof(double) * V);
  if (swing)
    memcpy(swing, s->swinging, sizeof(double) * V);
  if (traction)
    memcpy(traction, s->traction, sizeof(double) * V);
  if (applied)
    memcpy(applied, s->appliedDisp, sizeof(double) * 2 * V);
  if (scalars) {
    scalars[0] = s->globalSpeed;
    scalars[1] = s->speedEfficiency;
    scalars[2] = (double)s->iteration;
    scalars[3] = s->lastMaxDisplacement;
    scalars[4] = s->meanDegreePlusOne;
  }
}

static const char *kStatNames[5] = {
    "forceEmbedder.maxDisp", "forceEmbedder.speed",
    "forceEmbedder.attractiveForce", "forceEmbedder.repulsiveForce",
    "forceEmbedder.gravityForce"};

size_t ref_get_stats(refLayout *r, int which, double *out, size_t cap) {
  if (which < 0 || which > 4)
    return 0;
  const gvizStatSeries *ser =
      gvizEmbeddedGraphFindStatSeries((gvizEmbeddedGraph *)&r->s, kStatNames[which]);
  if (!ser)
    return 0;
  size_t n = ser->count < cap ? ser->count : cap;
  if (out)
    memcpy(out, ser->samples, sizeof(double) * n);
  return ser->count;
}

void ref_release(refLayout *r) {
  if (!r)
    return;
  gvizForceEmbedderRelease(&r->s);
  gvizGraphRelease(&r->g);
  free(r);
}

/* ---------------------------------------------------------------------- */
/* quadtree dumps (paths are 2-bit quadrant digits, MSB first)              */
/* ---------------------------------------------------------------------- */

static void put_digit(uint64_t *hi, uint64_t *lo, int depth, int q) {
  if (depth <= 32)
    *hi |= (uint64_t)q << (2 * (32 - depth));
  else if (depth <= 64)
    *lo |= (uint64_t)q << (2 * (64 - depth));
}

typedef struct leafCtx {
  int32_t *leafDepth;
  uint64_t *pathHi, *pathLo;
  size_t nodes;
  /* node dump */
  size_t cap, w;
  int32_t *nDepth, *nLeaf;
  uint64_t *nHi, *nLo, *nCount;
  double *nMass, *nComX, *nComY;
} leafCtx;

static uint64_t walk_leaves(const gvizQuadtreeNode *nd, int depth, uint64_t hi,
                            uint64_t lo, leafCtx *c) {
  if (!nd)
    return 0;
  c->nodes++;
  uint64_t cnt = 0;
  size_t slot = (size_t)-1;
  if (c->nDepth && c->w < c->cap)
    slot = c->w++;
  if (gvizQuadtreeNodeIsLeaf(nd)) {
    size_t n = gvizQuadtreeNodePointCount(nd);
    for (size_t i = 0; i < n; i++) {
      size_t idx = gvizQuadtreeNodePointAt(nd, i);
      if (c->leafDepth) {
        c->leafDepth[idx] = depth;
        c->pathHi[idx] = hi;
        c->pathLo[idx] = lo;
      }
    }
    cnt = n;
  } else {
    for (int q = 0; q < GVIZ_QUAD_COUNT; q++) {
      uint64_t h2 = hi, l2 = lo;
      put_digit(&h2, &l2, depth + 1, q);
      cnt += walk_leaves(gvizQuadtreeNodeChild(nd, (gvizQuadrant)q), depth + 1,
                         h2, l2, c);
    }
  }
  if (slot != (size_t)-1) {
    double cx, cy;
    gvizQuadtreeNodeCenterOfMass(nd, &cx, &cy);
    c->nDepth[slot] = depth;
    c->nHi[slot] = hi;
    c->nLo[slot] = lo;
    c->nMass[slot] = nd->mass;
    c->nComX[slot] = cx;
    c->nComY[slot] = cy;
    c->nLeaf[slot] = gvizQuadtreeNodeIsLeaf(nd);
    c->nCount[slot] = cnt;
  }
  return cnt;
}

int ref_quadtree_leaves(const double *pts, const double *mass, size_t n,
                        size_t k, int32_t *leafDepth, uint64_t *pathHi,
                        uint64_t *pathLo, size_t *nodeCountOut) {
  gvizQuadtree t;
  if (gvizQuadtreeInit(&t, pts, mass, n, k) != 0) {
    gvizQuadtreeRelease(&t);
    return -1;
  }
  leafCtx c;
  memset(&c, 0, sizeof(c));
  c.leafDepth = leafDepth;
  c.pathHi = pathHi;
  c.pathLo = pathLo;
  walk_leaves(gvizQuadtreeRoot(&t), 0, 0, 0, &c);
  if (nodeCountOut)
    *nodeCountOut = c.nodes;
  gvizQuadtreeRelease(&t);
  return 0;
}

/* All nodes with a non-empty subtree, in DFS order. Returns how many. */
size_t ref_quadtree_nodes(const double *pts, const double *mass, size_t n,
                          size_t k, size_t cap, int32_t *depth,
                          uint64_t *pathHi, uint64_t *pathLo, double *outMass,
                          double *comX, double *comY, int32_t *isLeaf,
                          uint64_t *count) {
  gvizQuadtree t;
  if (gvizQuadtreeInit(&t, pts, mass, n, k) != 0) {
    gvizQuadtreeRelease(&t);
    return 0;
  }
  /* first pass: everything, then compact out empty subtrees */
  size_t total = t.nodesUsed;
  leafCtx c;
  memset(&c, 0, sizeof(c));
  c.cap = total;
  c.nDepth = malloc(sizeof(int32_t) * total);
  c.nLeaf = malloc(sizeof(int32_t) * total);
  c.nHi = malloc(sizeof(uint64_t) * total);
  c.nLo = malloc(sizeof(uint64_t) * total);
  c.nCount = malloc(sizeof(uint64_t) * total);
  c.nMass = malloc(sizeof(double) * total);
  c.nComX = malloc(sizeof(double) * total);
  c.nComY = malloc(sizeof(double) * total);
  walk_leaves(gvizQuadtreeRoot(&t), 0, 0, 0, &c);
  size_t w = 0;
  for (size_t i = 0; i < c.w && w < cap; i++) {
    if (c.nCount[i] == 0)
      continue;
    depth[w] = c.nDepth[i];
    pathHi[w] = c.nHi[i];
    pathLo[w] = c.nLo[i];
    outMass[w] = c.nMass[i];
    comX[w] = c.nComX[i];
    comY[w] = c.nComY[i];
    isLeaf[w] = c.nLeaf[i];
    count[w] = c.nCount[i];
    w++;
  }
  free(c.nDepth);
  free(c.nLeaf);
  free(c.nHi);
  free(c.nLo);
  free(c.nCount);
  free(c.nMass);
  free(c.nComX);
  free(c.nComY);
  gvizQuadtreeRelease(&t);
  return w;
}

/* ---------------------------------------------------------------------- */
/* CPU timing helpers for the baseline                                     */
/* ---------------------------------------------------------------------- */

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* Runs `steps` reference steps, writing each step's wall time (s). */
void ref_time_steps(refLayout *r, int steps, double *secondsOut) {
  for (int i = 0; i < steps; i++) {
    double t0 = now_s();
    gvizForceEmbedderStep(&r->s);
    secondsOut[i] = now_s() - t0;
  }
}

/* Worker count gvizThreadPoolCreate(0) uses (src/core/gvizThreadPool.c:75-78). */
long ref_pool_threads(void) { return sysconf(_SC_NPROCESSORS_ONLN); }

/* The reference's own loaders (src/utils/graphLoader.c), exported as CSR
 * from the loaded graph's adjacency lists (neighbour order as the subgraph
 * neighbour iterator yields it). Returns the vertex count and *entries, or
 * -1 when the loader fails. With row == NULL only the sizes are returned. */
static long long csr_of_graph(gvizGraph *g, uint64_t *row, uint32_t *col, size_t *entries) {
  const size_t V = gvizGraphSize(g);
  size_t off = 0;
  for (size_t i = 0; i < V; i++) {
    gvizArray *nb = gvizGraphGetVertexNeighbors(g, i);
    if (row)
      row[i] = off;
    for (size_t k = 0; k < nb->count; k++) {
      if (col)
        col[off] = (uint32_t)*(size_t *)gvizArrayAtIndex(nb, k);
      off++;
    }
  }
  if (row)
    row[V] = off;
  *entries = off;
  return (long long)V;
}

long long ref_load_edges_csr(const char *path, int directed, int skipHeader,
                             uint64_t *row, uint32_t *col, size_t *entries) {
  gvizEdgesFileOptions o;
  gvizEdgesFileOptionsInit(&o);
  o.directed = directed;
  o.skip_header = skipHeader;
  gvizGraph g;
  if (gvizGraphLoadFromEdgesFile(path, &o, &g) < 0)
    return -1;
  long long V = csr_of_graph(&g, row, col, entries);
  gvizGraphRelease(&g);
  return V;
}

long long ref_load_obj_csr(const char *path, uint64_t *row, uint32_t *col, size_t *entries) {
  gvizGraph g;
  if (gvizGraphLoadFromObjFile(path, &g) < 0)
    return -1;
  long long V = csr_of_graph(&g, row, col, entries);
  gvizGraphRelease(&g);
  return V;
}

long long ref_load_gexf_csr(const char *path, uint64_t *row, uint32_t *col, size_t *entries) {
  gvizGraph g;
  if (gvizGraphLoadFromGexfFile(path, &g) < 0)
    return -1;
  long long V = csr_of_graph(&g, row, col, entries);
  gvizGraphFreeVertexDataStrings(&g);
  gvizGraphRelease(&g);
  return V;
}

/* gviz's own text embedding load / save on the embedder's graph. */
int ref_load_embedding(refLayout *r, const char *path) {
  return gvizEmbeddedGraphLoadEmbedding((gvizEmbeddedGraph *)&r->s, path);
}

int ref_save_embedding(refLayout *r, const char *name, const char *path) {
  return gvizEmbeddedGraphSaveEmbedding((gvizEmbeddedGraph *)&r->s, name, path);
}

/* ---------------------------------------------------------------------- */
/* GRIP (src/embedders/gvizGRIPEmbedder.c), 2-D, full subgraph: the        */
/* reference's own Begin / NextStage / RefineRound, with its filtration,   */
/* k-nearest lists, positions and heat read back for the device round.    */
/* ---------------------------------------------------------------------- */
#include "core/gvizThreadPool.h"
#include "ds/gvizArray.h"
#include "embedders/gvizGRIPEmbedder.h"

typedef struct refGrip {
  gvizGraph g;
  gvizGRIPState s;
  int initRes;
} refGrip;

/* serial != 0 runs the reference's parallel phases on the calling thread
 * (its own NULL-pool fallback, src/embedders/gvizGRIPEmbedder.c:310-311):
 * refinementPass1Range (:1081-1083) sets the dispCalculated bits of one
 * word from several pool threads without atomics, so with the pool a
 * vertex can lose its mark and restart at heat L/6 in the next round, which
 * makes pooled rounds irreproducible. */
refGrip *ref_grip_create(size_t V, const uint32_t *ea, const uint32_t *eb, size_t E,
                         int serial) {
  refGrip *r = calloc(1, sizeof(refGrip));
  if (!r)
    return NULL;
  gvizGraphInitAtCapacity(&r->g, 0, V ? V : 1);
  for (size_t i = 0; i < V; i++)
    gvizGraphAddVertex(&r->g, NULL, NULL, NULL);
  for (size_t e = 0; e < E; e++)
    gvizGraphAddEdge(&r->g, ea[e], eb[e]);
  gvizGraphBuildLayout(&r->g);
  gvizSubgraph sg = gvizSubgraphCreateFull(&r->g);
  gvizGRIPEmbedderConfigureStats(&r->s, false);
  r->initRes = gvizGRIPEmbedderInit(&r->s, sg, 0, 2);
  if (serial && r->initRes == 0) {
    gvizThreadPoolDestroy(r->s.pool);
    r->s.pool = NULL;
  }
  return r;
}

int ref_grip_init_result(refGrip *r) { return r->initRes; }
/* gvizGRIPEmbedderInit allocates the BFS stamp array without clearing it
 * (src/embedders/gvizGRIPEmbedder.c:253) and Begin's MIS filtration reads it
 * (:511 gripPickFarCandidate, :603 verticesWithinRadius) as if every stamp
 * were older than the first epoch, so leftover heap contents could mark
 * vertices visited and two identical states could build different
 * filtrations. Zeroed first, as the epoch scheme assumes (Begin clears it
 * the same way when the epoch wraps, :605-607). */
void ref_grip_begin(refGrip *r) {
  if (r->s.radiusBfsStamp)
    memset(r->s.radiusBfsStamp, 0, sizeof(size_t) * gvizGraphSize(&r->g));
  gvizGRIPEmbedderBegin(&r->s);
}
void ref_grip_next_stage(refGrip *r) { gvizGRIPEmbedderNextStage(&r->s); }
size_t ref_grip_layer(refGrip *r) { return r->s.currLayer; }
size_t ref_grip_layer_count(refGrip *r) { return r->s.layerCount; }

/* the active vertices of the current layer, in filtration order */
size_t ref_grip_active(refGrip *r, uint32_t *out, size_t cap) {
  const size_t n = *(const size_t *)gvizArrayAtIndex(&r->s.misBorder, r->s.currLayer);
  for (size_t i = 0; i < n && i < cap; i++)
    out[i] = (uint32_t)r->s.misFiltration[i];
  return n;
}

/* each active vertex's k-nearest list (vertex, graph distance), CSR over
 * the filtration order; returns the total entries */
size_t ref_grip_knn(refGrip *r, uint64_t *off, uint32_t *v, uint32_t *dist, size_t cap) {
  const size_t n = *(const size_t *)gvizArrayAtIndex(&r->s.misBorder, r->s.currLayer);
  size_t k = 0;
  for (size_t i = 0; i < n; i++) {
    const gvizGRIPDecorators *d = r->s.dec + r->s.misFiltration[i];
    if (off)
      off[i] = k;
    for (size_t j = 0; j < d->knn.count; j++, k++) {
      if (k < cap) {
        const gvizFoundVertex *f = (const gvizFoundVertex *)gvizArrayAtIndex(&d->knn, j);
        v[k] = (uint32_t)f->v;
        dist[k] = (uint32_t)f->dist;
      }
    }
  }
  if (off)
    off[n] = k;
  return k;
}

/* one refinement round; stats = {maxDisplacement, meanDisplacement, meanForce} */
void ref_grip_refine(refGrip *r, double *stats) {
  gvizGRIPEmbedderRefineRound(&r->s);
  const gvizGRIPRoundStats st = gvizGRIPEmbedderLastRoundStats(&r->s);
  stats[0] = st.maxDisplacement;
  stats[1] = st.meanDisplacement;
  stats[2] = st.meanForce;
}

void ref_grip_get_positions(refGrip *r, double *xy) {
  gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)&r->s;
  const size_t V = gvizGraphSize(&r->g);
  for (size_t i = 0; i < V; i++) {
    const double *p = gvizEmbeddedGraphGetVPosition(eg, i);
    xy[2 * i] = p[0];
    xy[2 * i + 1] = p[1];
  }
}

void ref_grip_set_positions(refGrip *r, const double *xy) {
  gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)&r->s;
  const size_t V = gvizGraphSize(&r->g);
  for (size_t i = 0; i < V; i++) {
    double p[2] = {xy[2 * i], xy[2 * i + 1]};
    gvizEmbeddedGraphSetVPosition(eg, i, p);
  }
}

/* per vertex: heat, last displacement (2), previous cosine */
void ref_grip_get_decorators(refGrip *r, double *heat, double *disp, double *oldCos) {
  const size_t V = gvizGraphSize(&r->g);
  for (size_t i = 0; i < V; i++) {
    heat[i] = r->s.dec[i].heat;
    disp[2 * i] = r->s.dec[i].disp[0];
    disp[2 * i + 1] = r->s.dec[i].disp[1];
    oldCos[i] = r->s.dec[i].oldCos;
  }
}

void ref_grip_release(refGrip *r) {
  if (!r)
    return;
  gvizGRIPEmbedderRelease(&r->s);
  gvizGraphRelease(&r->g);
  free(r);
}

/* the state, for gviz-side glue that attaches to it */
void *ref_grip_state(refGrip *r) { return &r->s; }

/* "grip.refineRound" through the action registry, as a front-end invokes it */
int ref_grip_invoke_refine(refGrip *r) {
  return gvizEmbeddedGraphInvokeAction((gvizEmbeddedGraph *)&r->s, "grip.refineRound", NULL);
}

/* lastRoundStats {max, mean displacement, mean force} and currRound */
size_t ref_grip_last_stats(refGrip *r, double *stats) {
  stats[0] = r->s.lastRoundStats.maxDisplacement;
  stats[1] = r->s.lastRoundStats.meanDisplacement;
  stats[2] = r->s.lastRoundStats.meanForce;
  return r->s.currRound;
}
