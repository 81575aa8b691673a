/*
 * gvizCudaForceEmbedder.c -- gviz-side glue for libgvizcuda (C11). A gviz
 * maintainer adds this file to the gviz library; see
 * include/gvizCudaForceEmbedder.h for the contract.
 *
 * It only uses gviz's public API: the embedder state fields, the subgraph
 * neighbour iterator (src/ds/gvizSubgraph.c:466-519) to build CSR in compact
 * order, the position accessors (src/embedders/gvizEmbeddedGraph.c:389-404),
 * the action registry (:222-293) and the stat series (:332-357).
 */
#include "gvizCudaForceEmbedder.h"

#include <stdlib.h>
#include <string.h>

#include "ds/gvizGraph.h"
#include "ds/gvizSubgraph.h"
#include "embedders/gvizEmbeddedGraph.h"
#include "embedders/gvizForceModel.h"

typedef struct attached {
  gvizForceEmbedderState *state;
  gvizCudaForce *h;
  gvizCudaOptions opt;
  double *xy;              /* compact positions, 2V */
  size_t lastIteration;    /* state->iteration after our last step */
  int lastError;
  int farWanted;           /* the caller turned the learned walk on (handle) */
  int farPushed;           /* farField as this glue last pushed it */
  struct attached *next;
} attached;

static attached *g_attached = NULL;

static attached *find(const gvizForceEmbedderState *state) {
  for (attached *a = g_attached; a; a = a->next)
    if (a->state == state)
      return a;
  return NULL;
}

static void gather(attached *a) {
  gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)a->state;
  for (size_t i = 0; i < a->state->vertexCount; i++) {
    double *p = gvizEmbeddedGraphGetVPosition(eg, a->state->vertices[i]);
    a->xy[2 * i] = p[0];
    a->xy[2 * i + 1] = p[1];
  }
}

static void scatter(attached *a) {
  gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)a->state;
  for (size_t i = 0; i < a->state->vertexCount; i++) {
    double p[2] = {a->xy[2 * i], a->xy[2 * i + 1]};
    gvizEmbeddedGraphSetVPosition(eg, a->state->vertices[i], p);
  }
}

static void state_params(const gvizForceEmbedderState *s, const gvizCudaOptions *o,
                         gvizCudaForceParams *out) {
  gvizCudaForceParams p;
  gvizCudaForceDefaultParams(&p);
  p.edgeLength = s->edgeLength;
  p.theta = s->theta;
  p.nodesPerCell = (uint32_t)s->nodesPerCell;
  p.barnesHutEnabled = s->barnesHutEnabled;
  p.gravityK = s->gravityK;
  p.radiusBase = s->radiusBase;
  p.radiusPerDegree = s->radiusPerDegree;
  p.overlapConstant = s->overlapConstant;
  p.preventOverlap = s->preventOverlap;
  p.precision = o->precision;
  p.jitterTolerance = s->jitterTolerance;
  p.strictReductions = o->strictReductions;
  *out = p;
}

static int32_t state_model(const gvizForceEmbedderState *s) {
  return s->model == gvizForceModelGet(GVIZ_FORCE_MODEL_LINLOG) ? GVIZ_CUDA_MODEL_LINLOG
                                                                : GVIZ_CUDA_MODEL_FR;
}

/* Configuration is re-read before every step: the toggle action and the
 * Configure* setters may run between steps. The learned far-field options
 * have no embedder field; whatever the caller set on the handle
 * (gvizCudaForceEmbedderHandle) is kept, except that the learned walk
 * (FP32 Barnes-Hut only) is held off while the embedder has Barnes-Hut
 * off (gvizForceEmbedderSetBarnesHutEnabled,
 * src/embedders/gvizForceEmbedder.c:381) or the glue runs FP64: the step then
 * takes the exact or the FP64 walk, as the reference would, and the learned
 * walk comes back with Barnes-Hut. When something else turns it off (the
 * caller, or the handle's judge falling back to the plain walk), it stays
 * off. */
static int push_params(attached *a) {
  const gvizForceEmbedderState *s = a->state;
  gvizCudaForceParams p;
  gvizCudaForceDefaultParams(&p);
  p.edgeLength = s->edgeLength;
  p.theta = s->theta;
  p.nodesPerCell = (uint32_t)s->nodesPerCell;
  p.barnesHutEnabled = s->barnesHutEnabled;
  p.gravityK = s->gravityK;
  p.radiusBase = s->radiusBase;
  p.radiusPerDegree = s->radiusPerDegree;
  p.overlapConstant = s->overlapConstant;
  p.preventOverlap = s->preventOverlap;
  p.precision = a->opt.precision;
  p.jitterTolerance = s->jitterTolerance;
  p.strictReductions = a->opt.strictReductions;
  gvizCudaForceParams cur;
  if (gvizCudaForceGetParams(a->h, &cur) != GVIZ_CUDA_OK)
    return gvizCudaForceSetParams(a->h, &p);
  if (cur.farField)
    a->farWanted = 1;
  else if (a->farPushed)
    a->farWanted = 0; /* turned off since our last push */
  p.farField = (a->farWanted && p.barnesHutEnabled && p.precision == GVIZ_CUDA_FP32) ? 1 : 0;
  a->farPushed = p.farField;
  p.farGroupSpread = cur.farGroupSpread;
  p.farCellGroups = cur.farCellGroups;
  p.farHubTargets = cur.farHubTargets;
  p.farHubTheta = cur.farHubTheta;
  if (memcmp(&cur, &p, sizeof(p)) == 0)
    return GVIZ_CUDA_OK;
  return gvizCudaForceSetParams(a->h, &p);
}

/* Re-uploads the FA2 history when something other than this glue moved the
 * state (Begin, or CPU steps in between). */
static int push_fa2(attached *a, int force) {
  gvizForceEmbedderState *s = a->state;
  if (force || s->iteration == 0 || s->iteration != a->lastIteration)
    return gvizCudaForceSetFa2State(a->h, s->structForce, &s->globalSpeed,
                                    &s->speedEfficiency);
  return gvizCudaForceSetFa2State(a->h, NULL, &s->globalSpeed,
                                  &s->speedEfficiency);
}

static const char *kStat[5] = {
    "forceEmbedder.maxDisp", "forceEmbedder.speed",
    "forceEmbedder.attractiveForce", "forceEmbedder.repulsiveForce",
    "forceEmbedder.gravityForce"};

static void append_stats(gvizForceEmbedderState *s, const double *row) {
  for (int q = 0; q < 5; q++)
    gvizEmbeddedGraphStatAppend((gvizEmbeddedGraph *)s, kStat[q], row[q]);
}

static int pull_state(attached *a) {
  gvizForceEmbedderState *s = a->state;
  int rc = gvizCudaForceGetFa2State(a->h, a->opt.syncScratch ? s->structForce : NULL,
                                    &s->globalSpeed, &s->speedEfficiency);
  if (rc == GVIZ_CUDA_OK && a->opt.syncScratch)
    rc = gvizCudaForceGetForces(a->h, s->disp, NULL, s->attForceMag, s->repForceMag,
                                s->swinging, s->traction, s->appliedDisp);
  return rc;
}

static void gpu_step_action(gvizEmbeddedGraph *embedding, void *userData,
                            const gvizActionPayload *payload) {
  (void)userData;
  (void)payload;
  gvizForceEmbedderState *state = (gvizForceEmbedderState *)embedding;
  if (!state->begun)
    return;
  gvizCudaForceEmbedderStep(state);
}

static void cpu_step_action(gvizEmbeddedGraph *embedding, void *userData,
                            const gvizActionPayload *payload) {
  (void)userData;
  (void)payload;
  gvizForceEmbedderState *state = (gvizForceEmbedderState *)embedding;
  if (!state->begun)
    return;
  gvizForceEmbedderStep(state);
}

/* CSR of one embedder's subgraph in compact order: row[V+1] (offsets start
 * at `base`, for concatenating graphs), deg[V] and *col (allocated here;
 * neighbour indices are compact within this state). Neighbours come from
 * the subgraph neighbour iterator, so duplicates and both directions are
 * kept as gviz stores them. */
static int state_csr(const gvizForceEmbedderState *state, uint64_t base, uint64_t *row,
                     uint64_t *deg, uint32_t **col) {
  const gvizEmbeddedGraph *eg = (const gvizEmbeddedGraph *)state;
  const size_t V = state->vertexCount;
  const size_t n = gvizGraphSize(eg->subgraph.g);
  size_t *compact = malloc(sizeof(size_t) * (n ? n : 1));
  if (!compact)
    return GVIZ_CUDA_ERR_ALLOC;
  for (size_t i = 0; i < n; i++)
    compact[i] = (size_t)-1;
  for (size_t i = 0; i < V; i++)
    compact[state->vertices[i]] = i;
  uint64_t off = 0;
  for (size_t i = 0; i < V; i++) {
    row[i] = base + off;
    deg[i] = state->degree[i];
    gvizSubgraphNeighborIterator it = gvizSubgraphNeighborIteratorCreate(
        (gvizSubgraph *)&eg->subgraph, state->vertices[i]);
    size_t u;
    while (gvizSubgraphNeighborIterate(&it, &u))
      off++;
  }
  row[V] = base + off;
  *col = malloc(sizeof(uint32_t) * (off ? off : 1));
  int rc = *col ? GVIZ_CUDA_OK : GVIZ_CUDA_ERR_ALLOC;
  for (size_t i = 0, e = 0; rc == GVIZ_CUDA_OK && i < V; i++) {
    gvizSubgraphNeighborIterator it = gvizSubgraphNeighborIteratorCreate(
        (gvizSubgraph *)&eg->subgraph, state->vertices[i]);
    size_t u;
    while (gvizSubgraphNeighborIterate(&it, &u)) {
      if (compact[u] == (size_t)-1) {  /* neighbour outside the subgraph */
        rc = GVIZ_CUDA_ERR_ARG;
        break;
      }
      (*col)[e++] = (uint32_t)compact[u];
    }
  }
  free(compact);
  return rc;
}

int gvizCudaForceAttach(gvizForceEmbedderState *state,
                        const gvizCudaOptions *options) {
  if (!state)
    return GVIZ_CUDA_ERR_ARG;
  gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)state;
  if (eg->embedding.dim != 2)
    return GVIZ_CUDA_ERR_DIMENSION;
  if (find(state))
    gvizCudaForceDetach(state);
  const size_t V = state->vertexCount;
  uint64_t *row = malloc(sizeof(uint64_t) * (V + 1));
  uint64_t *deg = malloc(sizeof(uint64_t) * (V ? V : 1));
  uint32_t *col = NULL;
  attached *a = calloc(1, sizeof(attached));
  int rc = (row && deg && a) ? GVIZ_CUDA_OK : GVIZ_CUDA_ERR_ALLOC;
  if (rc == GVIZ_CUDA_OK)
    rc = state_csr(state, 0, row, deg, &col);
  if (rc == GVIZ_CUDA_OK) {
    gvizCudaGraphDesc g;
    memset(&g, 0, sizeof(g));
    g.vertexCount = V;
    g.rowOffsets = row;
    g.neighbors = col;
    g.degree = deg;
    g.graphCount = 1;
    g.model = state->model == gvizForceModelGet(GVIZ_FORCE_MODEL_LINLOG)
                  ? GVIZ_CUDA_MODEL_LINLOG
                  : GVIZ_CUDA_MODEL_FR;
    g.device = options ? options->device : 0;
    rc = gvizCudaForceCreate(&a->h, &g);
  }
  free(row);
  free(deg);
  free(col);
  if (!a)
    return rc;
  if (rc == GVIZ_CUDA_OK) {
    a->xy = malloc(sizeof(double) * 2 * (V ? V : 1));
    if (!a->xy)
      rc = GVIZ_CUDA_ERR_ALLOC;
  }
  if (rc != GVIZ_CUDA_OK) {
    if (a->h)
      gvizCudaForceDestroy(a->h);
    free(a->xy);
    free(a);
    return rc;
  }
  a->state = state;
  if (options)
    a->opt = *options;
  else {
    a->opt.device = 0;
    a->opt.precision = GVIZ_CUDA_FP32;
    a->opt.syncScratch = 1;
    a->opt.strictReductions = 0;
  }
  a->lastIteration = (size_t)-1;  /* first step uploads the FA2 history */
  if ((rc = push_params(a)) != GVIZ_CUDA_OK || (rc = gvizCudaForceBegin(a->h)) != GVIZ_CUDA_OK) {
    gvizCudaForceDestroy(a->h);
    free(a->xy);
    free(a);
    return rc;
  }
  a->next = g_attached;
  g_attached = a;
  if (gvizEmbeddedGraphAddAction(eg, "forceEmbedder.step", gpu_step_action, a) < 0) {
    gvizCudaForceDetach(state);
    return GVIZ_CUDA_ERR_ALLOC;
  }
  return GVIZ_CUDA_OK;
}

double gvizCudaForceEmbedderStep(gvizForceEmbedderState *state) {
  attached *a = find(state);
  if (!a)
    return (double)GVIZ_CUDA_ERR_ARG;
  int rc = push_params(a);
  if (rc == GVIZ_CUDA_OK)
    rc = push_fa2(a, 0);
  if (rc != GVIZ_CUDA_OK) {
    a->lastError = rc;
    return (double)rc;
  }
  gather(a);
  gvizCudaStepStats st;
  double md = gvizCudaForceStepHost(a->h, a->xy, &st);
  if (md < 0.0) {
    a->lastError = (int)md;
    return md;
  }
  scatter(a);
  rc = pull_state(a);
  if (rc != GVIZ_CUDA_OK)
    a->lastError = rc;
  state->iteration++;
  state->lastMaxDisplacement = md;
  const double row[5] = {st.maxDisp, st.speed, st.meanAttractive,
                         st.meanRepulsive, st.meanGravity};
  append_stats(state, row);
  a->lastIteration = state->iteration;
  return md;
}

int gvizCudaForceEmbedderRun(gvizForceEmbedderState *state, size_t maxIters,
                             double epsilon) {
  attached *a = find(state);
  if (!a)
    return GVIZ_CUDA_ERR_ARG;
  if (!state->begun)
    return -1;
  int rc = push_params(a);
  if (rc == GVIZ_CUDA_OK)
    rc = push_fa2(a, 0);
  if (rc != GVIZ_CUDA_OK) {
    a->lastError = rc;
    return rc;
  }
  gather(a);
  int64_t before = gvizCudaForceStatHistory(a->h, 0, NULL, 0);
  uint64_t rounds = 0;
  if ((rc = gvizCudaForceSetPositions(a->h, a->xy)) == GVIZ_CUDA_OK)
    rc = gvizCudaForceRun(a->h, maxIters, epsilon, &rounds);
  if (rc == GVIZ_CUDA_OK)
    rc = gvizCudaForceGetPositions(a->h, a->xy);
  if (rc != GVIZ_CUDA_OK) {
    a->lastError = rc;
    return rc;
  }
  scatter(a);
  pull_state(a);
  int64_t after = gvizCudaForceStatHistory(a->h, 0, NULL, 0);
  double *rows = malloc(sizeof(double) * 5 * (size_t)(after > 0 ? after : 1));
  if (rows && after > 0) {
    gvizCudaForceStatHistory(a->h, 0, rows, (size_t)after);
    /* the device keeps the last GVIZ_STATS_CAP rows; before/after index it */
    int64_t first = after - (int64_t)rounds;
    if (first < 0)
      first = 0;
    for (int64_t r = first; r < after; r++)
      append_stats(state, rows + 5 * r);
    if (rounds)
      state->lastMaxDisplacement = rows[5 * (after - 1)];
  }
  (void)before;
  free(rows);
  state->iteration += (size_t)rounds;
  a->lastIteration = state->iteration;
  return (int)rounds;
}

void gvizCudaForceDetach(gvizForceEmbedderState *state) {
  attached **pp = &g_attached;
  while (*pp && (*pp)->state != state)
    pp = &(*pp)->next;
  attached *a = *pp;
  if (!a)
    return;
  *pp = a->next;
  gvizEmbeddedGraphAddAction((gvizEmbeddedGraph *)state, "forceEmbedder.step",
                             cpu_step_action, NULL);
  gvizCudaForceDestroy(a->h);
  free(a->xy);
  free(a);
}

int gvizCudaForceEmbedderLastError(const gvizForceEmbedderState *state) {
  const attached *a = find(state);
  return a ? a->lastError : GVIZ_CUDA_ERR_ARG;
}

gvizCudaForce *gvizCudaForceEmbedderHandle(const gvizForceEmbedderState *state) {
  const attached *a = find(state);
  return a ? a->h : NULL;
}

/* ---- batched Run over many embedders ------------------------------------ */

static const gvizCudaOptions kDefaultOptions = {0, GVIZ_CUDA_FP32, 1, 0};

int gvizCudaForceEmbedderRunBatch(gvizForceEmbedderState **states, size_t n,
                                  size_t maxIters, double epsilon,
                                  const gvizCudaOptions *options, uint64_t *rounds) {
  if (!states || n == 0 || n > 0xffffffffu)
    return GVIZ_CUDA_ERR_ARG;
  const gvizCudaOptions *o = options ? options : &kDefaultOptions;
  gvizCudaForceParams p0, pi;
  for (size_t i = 0; i < n; i++) {
    if (!states[i])
      return GVIZ_CUDA_ERR_ARG;
    if (!states[i]->begun)
      return -1;
    if (((gvizEmbeddedGraph *)states[i])->embedding.dim != 2)
      return GVIZ_CUDA_ERR_DIMENSION;
    state_params(states[i], o, i ? &pi : &p0);
    /* one handle runs one model and one configuration */
    if (i && (memcmp(&pi, &p0, sizeof(pi)) != 0 ||
              state_model(states[i]) != state_model(states[0])))
      return GVIZ_CUDA_ERR_ARG;
  }
  size_t V = 0;
  for (size_t i = 0; i < n; i++)
    V += states[i]->vertexCount;
  int rc = GVIZ_CUDA_OK;
  uint64_t *row = malloc(sizeof(uint64_t) * (V + 1));
  uint64_t *deg = malloc(sizeof(uint64_t) * (V ? V : 1));
  uint64_t *goff = malloc(sizeof(uint64_t) * (n + 1));
  uint32_t **cols = calloc(n, sizeof(uint32_t *));
  double *xy = malloc(sizeof(double) * 2 * (V ? V : 1));
  double *sf = malloc(sizeof(double) * 2 * (V ? V : 1));
  double *speed = malloc(sizeof(double) * n), *eff = malloc(sizeof(double) * n);
  uint64_t *r = rounds ? rounds : malloc(sizeof(uint64_t) * n);
  uint32_t *col = NULL;
  gvizCudaForce *h = NULL;
  if (!row || !deg || !goff || !cols || !xy || !sf || !speed || !eff || !r)
    rc = GVIZ_CUDA_ERR_ALLOC;
  /* concatenated CSR, positions and FA2 history, graph by graph */
  uint64_t adj = 0, vb = 0;
  for (size_t i = 0; rc == GVIZ_CUDA_OK && i < n; i++) {
    const size_t Vi = states[i]->vertexCount;
    goff[i] = vb;
    rc = state_csr(states[i], adj, row + vb, deg + vb, &cols[i]);
    if (rc != GVIZ_CUDA_OK)
      break;
    gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)states[i];
    for (size_t k = 0; k < Vi; k++) {
      const double *q = gvizEmbeddedGraphGetVPosition(eg, states[i]->vertices[k]);
      xy[2 * (vb + k)] = q[0];
      xy[2 * (vb + k) + 1] = q[1];
    }
    memcpy(sf + 2 * vb, states[i]->structForce, sizeof(double) * 2 * Vi);
    speed[i] = states[i]->globalSpeed;
    eff[i] = states[i]->speedEfficiency;
    adj = row[vb + Vi];
    vb += Vi;
  }
  if (rc == GVIZ_CUDA_OK) {
    goff[n] = V;
    row[V] = adj;
    if (adj > 0xffffffffull)
      rc = GVIZ_CUDA_ERR_LIMIT;
  }
  if (rc == GVIZ_CUDA_OK && !(col = malloc(sizeof(uint32_t) * (adj ? adj : 1))))
    rc = GVIZ_CUDA_ERR_ALLOC;
  for (size_t i = 0, vbase = 0; rc == GVIZ_CUDA_OK && i < n; i++) {
    const size_t Vi = states[i]->vertexCount;
    for (uint64_t e = row[vbase]; e < row[vbase + Vi]; e++)
      col[e] = (uint32_t)(vbase + cols[i][e - row[vbase]]);
    vbase += Vi;
  }
  if (rc == GVIZ_CUDA_OK) {
    gvizCudaGraphDesc g;
    memset(&g, 0, sizeof(g));
    g.vertexCount = V;
    g.rowOffsets = row;
    g.neighbors = col;
    g.degree = deg;
    g.graphCount = n;
    g.graphOffsets = n > 1 ? goff : NULL;
    g.model = state_model(states[0]);
    g.device = o->device;
    rc = gvizCudaForceCreate(&h, &g);
  }
  if (rc == GVIZ_CUDA_OK)
    rc = gvizCudaForceSetParams(h, &p0);
  if (rc == GVIZ_CUDA_OK)
    rc = gvizCudaForceSetPositions(h, xy);
  if (rc == GVIZ_CUDA_OK)
    rc = gvizCudaForceBegin(h);
  if (rc == GVIZ_CUDA_OK)
    rc = gvizCudaForceSetFa2State(h, sf, speed, eff);
  if (rc == GVIZ_CUDA_OK)
    rc = gvizCudaForceRun(h, maxIters, epsilon, r);
  if (rc == GVIZ_CUDA_OK)
    rc = gvizCudaForceGetPositions(h, xy);
  if (rc == GVIZ_CUDA_OK)
    rc = gvizCudaForceGetFa2State(h, sf, speed, eff);
  /* write back: positions, FA2 state, counters and each graph's stat rows
   * (the device keeps each graph's latest 4096 rows since Begin) */
  double *rows = NULL;
  if (rc == GVIZ_CUDA_OK && !(rows = malloc(sizeof(double) * 5 * 4096)))
    rc = GVIZ_CUDA_ERR_ALLOC;
  for (size_t i = 0, vbase = 0; rc == GVIZ_CUDA_OK && i < n; i++) {
    gvizForceEmbedderState *s = states[i];
    const size_t Vi = s->vertexCount;
    gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)s;
    for (size_t k = 0; k < Vi; k++) {
      double q[2] = {xy[2 * (vbase + k)], xy[2 * (vbase + k) + 1]};
      gvizEmbeddedGraphSetVPosition(eg, s->vertices[k], q);
    }
    s->globalSpeed = speed[i];
    s->speedEfficiency = eff[i];
    if (o->syncScratch)
      memcpy(s->structForce, sf + 2 * vbase, sizeof(double) * 2 * Vi);
    const int64_t kept = gvizCudaForceStatHistory(h, (uint32_t)i, rows, 4096);
    const int64_t got = kept < 4096 ? kept : 4096;
    const int64_t take = (int64_t)r[i] < got ? (int64_t)r[i] : got;
    for (int64_t q = got - take; q < got; q++)
      append_stats(s, rows + 5 * q);
    if (take > 0)
      s->lastMaxDisplacement = rows[5 * (got - 1)];
    s->iteration += (size_t)r[i];
    vbase += Vi;
  }
  if (rc == GVIZ_CUDA_OK && o->syncScratch) {
    double *d = malloc(sizeof(double) * 2 * (V ? V : 1));
    double *ap = malloc(sizeof(double) * 2 * (V ? V : 1));
    double *m4 = malloc(sizeof(double) * 4 * (V ? V : 1));
    if (d && ap && m4)
      rc = gvizCudaForceGetForces(h, d, NULL, m4, m4 + V, m4 + 2 * V, m4 + 3 * V, ap);
    else
      rc = GVIZ_CUDA_ERR_ALLOC;
    for (size_t i = 0, vbase = 0; rc == GVIZ_CUDA_OK && i < n; i++) {
      gvizForceEmbedderState *s = states[i];
      const size_t Vi = s->vertexCount;
      memcpy(s->disp, d + 2 * vbase, sizeof(double) * 2 * Vi);
      memcpy(s->appliedDisp, ap + 2 * vbase, sizeof(double) * 2 * Vi);
      memcpy(s->attForceMag, m4 + vbase, sizeof(double) * Vi);
      memcpy(s->repForceMag, m4 + V + vbase, sizeof(double) * Vi);
      memcpy(s->swinging, m4 + 2 * V + vbase, sizeof(double) * Vi);
      memcpy(s->traction, m4 + 3 * V + vbase, sizeof(double) * Vi);
      vbase += Vi;
    }
    free(d);
    free(ap);
    free(m4);
  }
  if (h)
    gvizCudaForceDestroy(h);
  for (size_t i = 0; cols && i < n; i++)
    free(cols[i]);
  free(cols);
  free(rows);
  free(row);
  free(deg);
  free(goff);
  free(col);
  free(xy);
  free(sf);
  free(speed);
  free(eff);
  if (!rounds)
    free(r);
  return rc;
}
