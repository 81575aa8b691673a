/*
 * gviz_oracle.c -- CPU restatement (FP64, single thread) of gviz's
 * force-directed layout step.
 *
 * THIS FILE IS TEST INFRASTRUCTURE. It is the checker that the CUDA path in
 * grapher_b200/csrc is compared against; it is never linked into, called by
 * or shipped with libgvizcuda. Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it.
 *
 * What it restates (file:line in the Pretz0za/Grapher tree):
 *   - insertion-order quadtree with running centre of mass, leaf capacity
 *     nodesPerCell, subdivide-and-redistribute on overflow and an overflow
 *     leaf once halfSize <= 1e-9: src/ds/gvizQuadtree.c:65-192
 *   - Barnes-Hut repulsion walk (mass==0 skip, pairwise leaves with self
 *     skip, opening test 2*halfSize/|com-v| < theta, NW,NE,SW,SE recursion):
 *     src/embedders/gvizForceEmbedder.c:35-74
 *   - exact all-pairs repulsion: src/embedders/gvizForceEmbedder.c:104-115
 *   - per-vertex force assembly, magnitudes, structForce, gravity:
 *     src/embedders/gvizForceEmbedder.c:76-126
 *   - FR and LinLog force models: src/embedders/gvizForceModel.c:5-52,
 *     src/embedders/gvizForceDirected.c:141-149
 *   - pair formulas: include/core/gvizVec.h:320-334 (FR att), 404-428 (FR rep),
 *     486-499 (LinLog att), 552-578 (LinLog rep), 636-647 (gravity)
 *   - swing/traction, global speed, per-vertex speed, step tail:
 *     src/embedders/gvizForceEmbedder.c:128-197, 445-495
 *
 * Every floating-point expression keeps the reference's operand order and is
 * compiled with -ffp-contract=off, so for non-coincident inputs the oracle is
 * bit-identical to the reference (pinned by tests/test_oracle.py against the
 * reference built from source and against tests/golden/).
 *
 * One deliberate difference: two exactly coincident points have no direction.
 * The reference hashes the two buffer ADDRESSES (include/core/gvizVec.h:385-394),
 * which no other implementation can reproduce. The oracle and the CUDA path
 * share a deterministic, antisymmetric direction instead (see coincident_dir):
 * a 256-entry unit-circle table indexed by a hash of the two vertex indices,
 * negated for the higher index so the pair separates. Only finiteness and the
 * saturated magnitude k^2*C (or m_v*m_u*C) are comparable with the reference
 * there, which is what tests/core/gvizVecTests.c:107-117 pins.
 */
#include "gviz_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MIN_HALF_SIZE 1e-9
#define ORC_MIN_MASS 1e-9
#define ORC_NUMERIC_EPS 1e-7
#define ORC_EFF_MIN 0.05
#define ORC_EFF_MAX 1.0
#define ORC_MAX_RISE 0.5

/* ------------------------------------------------------------------------ */
/* coincident direction table (shared definition with the CUDA path)         */
/* ------------------------------------------------------------------------ */

static double g_dirTable[2 * ORC_DIR_TABLE];
static int g_dirTableReady = 0;

void orc_dir_table(double *out) {
  /* cos/sin of 2*pi*k/256 from the host libm; libgvizcuda builds the same
   * table with the same call on the host and uploads it. */
  for (int k = 0; k < ORC_DIR_TABLE; k++) {
    double a = 2.0 * M_PI * (double)k / (double)ORC_DIR_TABLE;
    out[2 * k] = cos(a);
    out[2 * k + 1] = sin(a);
  }
}

static uint64_t mix64(uint64_t z) {
  z ^= z >> 30;
  z *= 0xbf58476d1ce4e5b9ULL;
  z ^= z >> 27;
  z *= 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return z;
}

void orc_coincident_dir(uint64_t self, uint64_t other, double *ux, double *uy) {
  if (!g_dirTableReady) {
    orc_dir_table(g_dirTable);
    g_dirTableReady = 1;
  }
  uint64_t lo = self < other ? self : other;
  uint64_t hi = self < other ? other : self;
  uint64_t h = mix64(lo * 0x9e3779b97f4a7c15ULL + mix64(hi + 0x632be59bd9b4e019ULL));
  int k = (int)(h >> 56);
  double c = g_dirTable[2 * k], s = g_dirTable[2 * k + 1];
  if (self > other) {
    c = -c;
    s = -s;
  }
  *ux = c;
  *uy = s;
}

/* ------------------------------------------------------------------------ */
/* pair formulas                                                             */
/* ------------------------------------------------------------------------ */

/* FR attraction, include/core/gvizVec.h:320-334 */
static void fr_att(const double *v, const double *u, double k, double *acc) {
  double dx = u[0] - v[0];
  double dy = u[1] - v[1];
  double dist = sqrt(dx * dx + dy * dy);
  if (dist < 1e-9)
    return;
  double s = dist / k;
  acc[0] += s * dx;
  acc[1] += s * dy;
}

/* LinLog attraction, include/core/gvizVec.h:486-499 */
static void ll_att(const double *v, const double *u, double *acc) {
  double dx = u[0] - v[0];
  double dy = u[1] - v[1];
  double dist = sqrt(dx * dx + dy * dy);
  if (dist < 1e-9)
    return;
  double s = log(1.0 + dist) / dist;
  acc[0] += s * dx;
  acc[1] += s * dy;
}

/* shared body of FR / LinLog repulsion (include/core/gvizVec.h:404-428 and
 * 552-578): magnitude numerator `num` (k^2 or m_v*m_u), surface gap, bounded
 * overlap branch, unit direction or the coincident fallback. */
static void rep_core(const double *v, const double *u, double num,
                     double radiusSum, double overlapC, uint64_t self,
                     uint64_t other, double *acc) {
  double dx = u[0] - v[0];
  double dy = u[1] - v[1];
  double distSq = dx * dx + dy * dy;
  double dist = sqrt(distSq);
  double gap = dist - radiusSum;
  double mag = gap > 0.0 ? num / gap : num * overlapC;
  double ux, uy;
  if (dist > 0.0) {
    ux = dx / dist;
    uy = dy / dist;
  } else {
    orc_coincident_dir(self, other, &ux, &uy);
  }
  acc[0] -= mag * ux;
  acc[1] -= mag * uy;
}

/* model->repulsive: src/embedders/gvizForceModel.c:15-23 (FR, pseudo-body
 * mass truncated to size_t, then mass * force added, gvizForceDirected.c:141-149)
 * and :39-46 (LinLog). */
static void repulsive(const orcParams *p, const double *v, const double *u,
                      double vMass, double oMass, double vRadius, double oRadius,
                      uint64_t self, uint64_t other, double *acc) {
  if (p->model == ORC_MODEL_FR) {
    double scratch[2] = {0.0, 0.0};
    double k = p->edgeLength;
    rep_core(v, u, k * k, vRadius + oRadius, p->overlapConstant, self, other,
             scratch);
    double m = (double)(size_t)oMass;
    acc[0] += m * scratch[0];
    acc[1] += m * scratch[1];
  } else {
    rep_core(v, u, vMass * oMass, vRadius + oRadius, p->overlapConstant, self,
             other, acc);
  }
}

static double vertex_radius(const orcParams *p, const uint64_t *degree,
                            size_t i) {
  if (!p->preventOverlap)
    return 0.0;
  return p->radiusBase * (1.0 + p->radiusPerDegree * sqrt((double)degree[i]));
}

/* ------------------------------------------------------------------------ */
/* insertion-order quadtree                                                  */
/* ------------------------------------------------------------------------ */

typedef struct {
  double cx, cy, h, comX, comY, mass;
  int64_t child[4]; /* -1 on leaves */
  size_t *pts;
  size_t count, cap;
  int depth;
  uint64_t pathHi, pathLo; /* quadrant digits, MSB first, 2 bits per level */
} orcNode;

typedef struct {
  orcNode *nodes;
  size_t used, alloc;
  const double *pts;
  const double *mass;
  size_t n, k;
  int64_t root;
  int failed;
} orcTree;

static int64_t node_new(orcTree *t, double cx, double cy, double h, int depth,
                        uint64_t pathHi, uint64_t pathLo) {
  if (t->used == t->alloc) {
    size_t na = t->alloc ? t->alloc * 2 : 1024;
    orcNode *grown = realloc(t->nodes, na * sizeof(orcNode));
    if (!grown) {
      t->failed = 1;
      return -1;
    }
    t->nodes = grown;
    t->alloc = na;
  }
  orcNode *nd = &t->nodes[t->used];
  memset(nd, 0, sizeof(*nd));
  nd->cx = cx;
  nd->cy = cy;
  nd->h = h;
  nd->child[0] = nd->child[1] = nd->child[2] = nd->child[3] = -1;
  nd->cap = t->k;
  nd->pts = t->k ? malloc(sizeof(size_t) * t->k) : NULL;
  nd->depth = depth;
  nd->pathHi = pathHi;
  nd->pathLo = pathLo;
  return (int64_t)t->used++;
}

/* gvizQuadtreeQuadrantFor, src/ds/gvizQuadtree.c:65-73 */
static int quadrant_for(const orcNode *nd, double px, double py) {
  int east = px >= nd->cx;
  int north = py >= nd->cy;
  if (north)
    return east ? 1 : 0;
  return east ? 3 : 2;
}

static void append_digit(uint64_t *hi, uint64_t *lo, int depth, int q) {
  /* depth = depth of the child (1-based digit position) */
  if (depth <= 32)
    *hi |= (uint64_t)q << (2 * (32 - depth));
  else if (depth <= 64)
    *lo |= (uint64_t)q << (2 * (64 - depth));
}

/* gvizQuadtreeSubdivide, src/ds/gvizQuadtree.c:75-92 */
static int subdivide(orcTree *t, int64_t ni) {
  double quarter = t->nodes[ni].h / 2.0;
  double off[4][2] = {{-quarter, quarter},
                      {quarter, quarter},
                      {-quarter, -quarter},
                      {quarter, -quarter}};
  for (int q = 0; q < 4; q++) {
    orcNode *nd = &t->nodes[ni];
    uint64_t hi = nd->pathHi, lo = nd->pathLo;
    append_digit(&hi, &lo, nd->depth + 1, q);
    int64_t c = node_new(t, nd->cx + off[q][0], nd->cy + off[q][1], quarter,
                         nd->depth + 1, hi, lo);
    if (c < 0)
      return -1;
    t->nodes[ni].child[q] = c;
  }
  return 0;
}

/* gvizQuadtreeInsertPoint, src/ds/gvizQuadtree.c:112-157 */
static int insert_point(orcTree *t, int64_t ni, size_t idx) {
  double px = t->pts[2 * idx];
  double py = t->pts[2 * idx + 1];
  double pm = t->mass[idx];
  orcNode *nd = &t->nodes[ni];
  double newMass = nd->mass + pm;
  if (newMass > ORC_MIN_MASS || newMass < -ORC_MIN_MASS) {
    nd->comX = (nd->comX * nd->mass + px * pm) / newMass;
    nd->comY = (nd->comY * nd->mass + py * pm) / newMass;
  }
  nd->mass = newMass;

  if (nd->child[0] >= 0)
    return insert_point(t, nd->child[quadrant_for(nd, px, py)], idx);

  if (nd->count < nd->cap) {
    nd->pts[nd->count++] = idx;
    return 0;
  }

  if (nd->h <= ORC_MIN_HALF_SIZE) {
    size_t nc = nd->cap ? nd->cap * 2 : 1;
    size_t *grown = realloc(nd->pts, sizeof(size_t) * nc);
    if (!grown)
      return -1;
    nd->pts = grown;
    nd->cap = nc;
    nd->pts[nd->count++] = idx;
    return 0;
  }

  if (subdivide(t, ni) != 0)
    return -1;
  nd = &t->nodes[ni];
  size_t held = nd->count;
  for (size_t i = 0; i < held; i++) {
    nd = &t->nodes[ni];
    size_t hIdx = nd->pts[i];
    double hx = t->pts[2 * hIdx], hy = t->pts[2 * hIdx + 1];
    if (insert_point(t, nd->child[quadrant_for(nd, hx, hy)], hIdx) != 0)
      return -1;
  }
  nd = &t->nodes[ni];
  nd->count = 0;
  return insert_point(t, nd->child[quadrant_for(nd, px, py)], idx);
}

static void tree_free(orcTree *t) {
  for (size_t i = 0; i < t->used; i++)
    free(t->nodes[i].pts);
  free(t->nodes);
  memset(t, 0, sizeof(*t));
}

/* gvizQuadtreeBuild, src/ds/gvizQuadtree.c:159-192 */
static int tree_build(orcTree *t, const double *pts, const double *mass,
                      size_t n, size_t k) {
  memset(t, 0, sizeof(*t));
  t->pts = pts;
  t->mass = mass;
  t->n = n;
  t->k = k;
  t->root = -1;
  if (n == 0)
    return 0;
  double minX = pts[0], maxX = pts[0];
  double minY = pts[1], maxY = pts[1];
  for (size_t i = 1; i < n; i++) {
    double x = pts[2 * i], y = pts[2 * i + 1];
    minX = x < minX ? x : minX;
    maxX = x > maxX ? x : maxX;
    minY = y < minY ? y : minY;
    maxY = y > maxY ? y : maxY;
  }
  double sx = maxX - minX, sy = maxY - minY;
  double span = sx > sy ? sx : sy;
  double halfSize = span > 0.0 ? span / 2.0 : 1.0;
  double cx = (minX + maxX) / 2.0;
  double cy = (minY + maxY) / 2.0;
  t->root = node_new(t, cx, cy, halfSize, 0, 0, 0);
  if (t->root < 0)
    return -1;
  for (size_t i = 0; i < n; i++)
    if (insert_point(t, t->root, i) != 0)
      return -1;
  return t->failed ? -1 : 0;
}

/* bhAccumulateRepulsion, src/embedders/gvizForceEmbedder.c:35-74 */
static void bh_walk(const orcTree *t, const orcParams *p, const uint64_t *degree,
                    int64_t ni, size_t self, double vRadius, const double *vPos,
                    double *acc, uint64_t *interactions) {
  if (ni < 0)
    return;
  const orcNode *nd = &t->nodes[ni];
  if (nd->mass == 0)
    return;
  if (nd->child[0] < 0) {
    for (size_t i = 0; i < nd->count; i++) {
      size_t idx = nd->pts[i];
      if (idx == self)
        continue;
      repulsive(p, vPos, t->pts + 2 * idx, t->mass[self], t->mass[idx],
                vRadius, vertex_radius(p, degree, idx), self, idx, acc);
      if (interactions)
        (*interactions)++;
    }
    return;
  }
  double dx = nd->comX - vPos[0];
  double dy = nd->comY - vPos[1];
  double dist = sqrt(dx * dx + dy * dy);
  double ratio = (2.0 * nd->h) / dist;
  if (ratio < p->theta) {
    double com[2] = {nd->comX, nd->comY};
    /* a pseudo-body is never coincident with v: the test above needs dist > 0 */
    repulsive(p, vPos, com, t->mass[self], nd->mass, vRadius, 0.0, self,
              self, acc);
    if (interactions)
      (*interactions)++;
    return;
  }
  for (int q = 0; q < 4; q++)
    bh_walk(t, p, degree, nd->child[q], self, vRadius, vPos, acc, interactions);
}

/* ------------------------------------------------------------------------ */
/* public: quadtree dumps                                                    */
/* ------------------------------------------------------------------------ */

int orc_quadtree_leaves(const double *pts, const double *mass, size_t n,
                        size_t k, int32_t *leafDepth, uint64_t *pathHi,
                        uint64_t *pathLo, size_t *nodeCountOut) {
  orcTree t;
  if (tree_build(&t, pts, mass, n, k) != 0) {
    tree_free(&t);
    return -1;
  }
  for (size_t i = 0; i < t.used; i++) {
    const orcNode *nd = &t.nodes[i];
    if (nd->child[0] >= 0)
      continue;
    for (size_t j = 0; j < nd->count; j++) {
      size_t idx = nd->pts[j];
      leafDepth[idx] = nd->depth;
      pathHi[idx] = nd->pathHi;
      pathLo[idx] = nd->pathLo;
    }
  }
  if (nodeCountOut)
    *nodeCountOut = t.used;
  tree_free(&t);
  return 0;
}

size_t orc_quadtree_nodes(const double *pts, const double *mass, size_t n,
                          size_t k, size_t cap, int32_t *depth,
                          uint64_t *pathHi, uint64_t *pathLo, double *outMass,
                          double *comX, double *comY, int32_t *isLeaf,
                          uint64_t *count) {
  orcTree t;
  if (tree_build(&t, pts, mass, n, k) != 0) {
    tree_free(&t);
    return 0;
  }
  /* subtree point counts via reverse creation order (children are created
   * after their parents) */
  uint64_t *cnt = calloc(t.used ? t.used : 1, sizeof(uint64_t));
  for (size_t ii = t.used; ii-- > 0;) {
    const orcNode *nd = &t.nodes[ii];
    if (nd->child[0] < 0)
      cnt[ii] = nd->count;
    else
      for (int q = 0; q < 4; q++)
        cnt[ii] += cnt[nd->child[q]];
  }
  size_t w = 0;
  for (size_t i = 0; i < t.used && w < cap; i++) {
    const orcNode *nd = &t.nodes[i];
    if (cnt[i] == 0)
      continue;
    depth[w] = nd->depth;
    pathHi[w] = nd->pathHi;
    pathLo[w] = nd->pathLo;
    outMass[w] = nd->mass;
    comX[w] = nd->comX;
    comY[w] = nd->comY;
    isLeaf[w] = nd->child[0] < 0;
    count[w] = cnt[i];
    w++;
  }
  free(cnt);
  tree_free(&t);
  return w;
}

/* ------------------------------------------------------------------------ */
/* public: forces and the step                                               */
/* ------------------------------------------------------------------------ */

/* computeForceRange, src/embedders/gvizForceEmbedder.c:76-126, for all i.
 * pos: 2V compact positions. Writes disp, structForce, attMag, repMag. */
int orc_forces(size_t V, const uint64_t *rowOff, const uint32_t *cols,
               const double *mass, const uint64_t *degree, const orcParams *p,
               const double *pos, double *disp, double *structForce,
               double *attMag, double *repMag, uint64_t *interactions) {
  orcTree t;
  memset(&t, 0, sizeof(t));
  t.root = -1;
  if (p->barnesHutEnabled) {
    if (tree_build(&t, pos, mass, V, p->nodesPerCell) != 0) {
      tree_free(&t);
      return -1;
    }
  }
  for (size_t i = 0; i < V; i++) {
    const double *vPos = pos + 2 * i;
    double attF[2] = {0.0, 0.0}, repF[2] = {0.0, 0.0};
    for (uint64_t e = rowOff[i]; e < rowOff[i + 1]; e++) {
      const double *uPos = pos + 2 * (size_t)cols[e];
      if (p->model == ORC_MODEL_FR)
        fr_att(vPos, uPos, p->edgeLength, attF);
      else
        ll_att(vPos, uPos, attF);
    }
    double vRadius = vertex_radius(p, degree, i);
    uint64_t inter = 0;
    if (p->barnesHutEnabled) {
      bh_walk(&t, p, degree, t.root, i, vRadius, vPos, repF, &inter);
    } else {
      for (size_t j = 0; j < V; j++) {
        if (j == i)
          continue;
        repulsive(p, vPos, pos + 2 * j, mass[i], mass[j], vRadius,
                  vertex_radius(p, degree, j), i, j, repF);
      }
      inter = V ? V - 1 : 0;
    }
    if (interactions)
      interactions[i] = inter;
    double f[2] = {0.0, 0.0};
    f[0] += 1.0 * attF[0];
    f[1] += 1.0 * attF[1];
    f[0] += 1.0 * repF[0];
    f[1] += 1.0 * repF[1];
    if (attMag)
      attMag[i] = sqrt(attF[0] * attF[0] + attF[1] * attF[1]);
    if (repMag)
      repMag[i] = sqrt(repF[0] * repF[0] + repF[1] * repF[1]);
    if (structForce) {
      structForce[2 * i] = f[0];
      structForce[2 * i + 1] = f[1];
    }
    double gravityMag = p->gravityK * (double)(degree[i] + 1);
    double gd = sqrt(vPos[0] * vPos[0] + vPos[1] * vPos[1]);
    if (!(gd < 1e-9)) {
      double s = gravityMag / gd;
      f[0] -= s * vPos[0];
      f[1] -= s * vPos[1];
    }
    disp[2 * i] = f[0];
    disp[2 * i + 1] = f[1];
  }
  tree_free(&t);
  return 0;
}

/* updateGlobalSpeed, src/embedders/gvizForceEmbedder.c:140-185 */
static void update_speed(size_t V, const double *swing, const double *traction,
                         double jitterTolerance, double *speed, double *eff) {
  double totalSwing = 0.0, totalTraction = 0.0;
  for (size_t i = 0; i < V; i++) {
    totalSwing += swing[i];
    totalTraction += traction[i];
  }
  if (totalTraction < ORC_NUMERIC_EPS)
    return;
  double n = (double)V;
  double estJT = 0.05 * sqrt(n);
  double minJT = sqrt(estJT);
  double maxJT = 10.0;
  double jt = jitterTolerance *
              fmax(minJT, fmin(maxJT, estJT * totalTraction / (n * n)));
  if (totalSwing / totalTraction > 2.0) {
    if (*eff > ORC_EFF_MIN)
      *eff *= 0.5;
    jt = fmax(jt, jitterTolerance);
  }
  double target = totalSwing > ORC_NUMERIC_EPS
                      ? jt * *eff * totalTraction / totalSwing
                      : *speed;
  if (totalSwing > jt * totalTraction) {
    if (*eff > ORC_EFF_MIN)
      *eff *= 0.7;
  } else if (*speed < 1000.0) {
    *eff *= 1.3;
  }
  if (*eff < ORC_EFF_MIN)
    *eff = ORC_EFF_MIN;
  else if (*eff > ORC_EFF_MAX)
    *eff = ORC_EFF_MAX;
  *speed += fmin(target - *speed, ORC_MAX_RISE * *speed);
}

/* gvizForceEmbedderStep, src/embedders/gvizForceEmbedder.c:445-495, with the
 * position store in compact order. pos (2V) is updated in place; structForce
 * (2V) holds the previous round's structForce on entry and this round's on
 * return; speedState = {globalSpeed, speedEfficiency} in/out. stats receives
 * {maxDisp, speed, meanAtt, meanRep, meanGrav}. Optional per-vertex outputs
 * may be NULL. */
double orc_step(size_t V, const uint64_t *rowOff, const uint32_t *cols,
                const double *mass, const uint64_t *degree, const orcParams *p,
                double *pos, double *structForce, double *speedState,
                double *stats, double *dispOut, double *attMagOut,
                double *repMagOut, double *swingOut, double *tractionOut,
                double *appliedOut) {
  size_t n2 = V ? 2 * V : 1, n1 = V ? V : 1;
  double *old = malloc(sizeof(double) * n2);
  double *disp = malloc(sizeof(double) * n2);
  double *att = malloc(sizeof(double) * n1);
  double *rep = malloc(sizeof(double) * n1);
  double *swing = malloc(sizeof(double) * n1);
  double *trac = malloc(sizeof(double) * n1);
  double *applied = malloc(sizeof(double) * n2);
  if (V)
    memcpy(old, structForce, sizeof(double) * 2 * V);
  orc_forces(V, rowOff, cols, mass, degree, p, pos, disp, structForce, att, rep,
             NULL);
  /* computeSwingTractionRange, .c:128-138 */
  for (size_t i = 0; i < V; i++) {
    double *f = structForce + 2 * i, *o = old + 2 * i;
    double d0 = f[0] - o[0], d1 = f[1] - o[1];
    double s0 = f[0] + o[0], s1 = f[1] + o[1];
    swing[i] = mass[i] * sqrt(d0 * d0 + d1 * d1);
    trac[i] = mass[i] * 0.5 * sqrt(s0 * s0 + s1 * s1);
  }
  update_speed(V, swing, trac, p->jitterTolerance, &speedState[0],
               &speedState[1]);
  double speed = speedState[0];
  /* applySpeedRange, .c:187-197 */
  for (size_t i = 0; i < V; i++) {
    double factor = speed / (1.0 + sqrt(speed * swing[i]));
    applied[2 * i] = disp[2 * i] * factor;
    applied[2 * i + 1] = disp[2 * i + 1] * factor;
  }
  /* step tail, .c:467-492 */
  double maxDisp = 0.0, sumAtt = 0.0, sumRep = 0.0, sumDegPlusOne = 0.0;
  for (size_t i = 0; i < V; i++) {
    double *a = applied + 2 * i;
    double nrm = sqrt(a[0] * a[0] + a[1] * a[1]);
    if (nrm > maxDisp)
      maxDisp = nrm;
    sumAtt += att[i];
    sumRep += rep[i];
    pos[2 * i] += 1.0 * a[0];
    pos[2 * i + 1] += 1.0 * a[1];
    sumDegPlusOne += (double)(degree[i] + 1);
  }
  if (stats) {
    stats[0] = maxDisp;
    stats[1] = speed;
    stats[2] = V ? sumAtt / V : 0.0;
    stats[3] = V ? sumRep / V : 0.0;
    /* meanDegreePlusOne is fixed at Init, src/embedders/gvizForceEmbedder.c:251-259 */
    stats[4] = p->gravityK * (V ? sumDegPlusOne / (double)V : 0.0);
  }
  if (dispOut)
    memcpy(dispOut, disp, sizeof(double) * 2 * V);
  if (attMagOut)
    memcpy(attMagOut, att, sizeof(double) * V);
  if (repMagOut)
    memcpy(repMagOut, rep, sizeof(double) * V);
  if (swingOut)
    memcpy(swingOut, swing, sizeof(double) * V);
  if (tractionOut)
    memcpy(tractionOut, trac, sizeof(double) * V);
  if (appliedOut)
    memcpy(appliedOut, applied, sizeof(double) * 2 * V);
  free(old);
  free(disp);
  free(att);
  free(rep);
  free(swing);
  free(trac);
  free(applied);
  return maxDisp;
}

/* Exact FP64 repulsion of `nTargets` selected vertices against all V
 * vertices (the BH-off loop of src/embedders/gvizForceEmbedder.c:104-115),
 * used to judge approximate walks. */
void orc_exact_repulsion(size_t V, const double *mass, const uint64_t *degree,
                         const orcParams *p, const double *pos,
                         const uint64_t *targets, size_t nTargets,
                         double *repOut) {
  for (size_t t = 0; t < nTargets; t++) {
    size_t i = (size_t)targets[t];
    double acc[2] = {0.0, 0.0};
    double vr = vertex_radius(p, degree, i);
    for (size_t j = 0; j < V; j++) {
      if (j == i)
        continue;
      repulsive(p, pos + 2 * i, pos + 2 * j, mass[i], mass[j], vr,
                vertex_radius(p, degree, j), i, j, acc);
    }
    repOut[2 * t] = acc[0];
    repOut[2 * t + 1] = acc[1];
  }
}

/* Single pair-formula entry points, for the known-answer vectors of
 * tests/core/gvizVecTests.c:66-117. */
void orc_pair_fr_att(const double *v, const double *u, double k, double *acc) {
  fr_att(v, u, k, acc);
}
void orc_pair_fr_rep(const double *v, const double *u, double k,
                     double radiusSum, double overlapC, double *acc) {
  rep_core(v, u, k * k, radiusSum, overlapC, 0, 1, acc);
}
void orc_pair_linlog_att(const double *v, const double *u, double *acc) {
  ll_att(v, u, acc);
}
void orc_pair_linlog_rep(const double *v, const double *u, double vm,
                         double om, double radiusSum, double overlapC,
                         double *acc) {
  rep_core(v, u, vm * om, radiusSum, overlapC, 0, 1, acc);
}
