/*
 * gvizCudaGripEmbedder.c -- gviz-side glue for libgvizcuda's GRIP rounds
 * (C11). A gviz maintainer adds this file to the gviz library; see
 * include/gvizCudaGripEmbedder.h for the contract.
 *
 * It only uses gviz's public API: the GRIP state fields
 * (include/embedders/gvizGRIPEmbedder.h:40-78), the subgraph neighbour
 * iterator (src/ds/gvizSubgraph.c:466-519) to build CSR over vertex ids, the
 * position accessors (src/embedders/gvizEmbeddedGraph.c:389-404), the
 * action registry (:222-293) and the stat series (:332-357).
 */
#include "gvizCudaGripEmbedder.h"

#include <stdlib.h>
#include <string.h>

#include "algorithms/search/gvizKNearest.h"
#include "ds/gvizArray.h"
#include "ds/gvizBitArray.h"
#include "ds/gvizGraph.h"
#include "ds/gvizSubgraph.h"
#include "embedders/gvizEmbeddedGraph.h"

typedef struct gripAttached {
  gvizGRIPState *state;
  gvizCudaGrip *h;
  size_t V;
  size_t layer, active;  /* the layer the GPU holds (SIZE_MAX: none) */
  size_t rounds;         /* GPU rounds run on that layer */
  double *xy;            /* 2V positions scratch */
  int lastError;
  struct gripAttached *next;
} gripAttached;

static gripAttached *g_grip = NULL;

static gripAttached *grip_find(const gvizGRIPState *state) {
  for (gripAttached *a = g_grip; a; a = a->next)
    if (a->state == state) return a;
  return NULL;
}

static size_t grip_active_count(const gvizGRIPState *s) {
  return *(const size_t *)gvizArrayAtIndex((gvizArray *)&s->misBorder, s->currLayer);
}

static void grip_gpu_action(gvizEmbeddedGraph *embedding, void *userData,
                            const gvizActionPayload *payload) {
  (void)userData;
  (void)payload;
  gvizCudaGripEmbedderRefineRound((gvizGRIPState *)embedding);
}

static void grip_cpu_action(gvizEmbeddedGraph *embedding, void *userData,
                            const gvizActionPayload *payload) {
  (void)userData;
  (void)payload;
  gvizGRIPState *state = (gvizGRIPState *)embedding;
  if (state->layerCount == 0) return;
  gvizGRIPEmbedderRefineRound(state);
}

int gvizCudaGripAttach(gvizGRIPState *state, int32_t device, int32_t strictReductions) {
  if (!state) return GVIZ_CUDA_ERR_ARG;
  gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)state;
  if (eg->embedding.dim != 2) return GVIZ_CUDA_ERR_DIMENSION;
  if (grip_find(state)) return GVIZ_CUDA_OK;
  const size_t V = gvizGraphSize(eg->subgraph.g);
  uint64_t *row = calloc(V + 1, sizeof(uint64_t));
  size_t cap = 1024, n = 0;
  uint32_t *col = malloc(cap * sizeof(uint32_t));
  gripAttached *a = calloc(1, sizeof(gripAttached));
  double *xy = malloc((V ? 2 * V : 1) * sizeof(double));
  if (!row || !col || !a || !xy) {
    free(row), free(col), free(a), free(xy);
    return GVIZ_CUDA_ERR_ALLOC;
  }
  for (size_t v = 0; v < V; v++) {
    row[v] = n;
    if (!gvizSubgraphHasVertex(&eg->subgraph, v)) continue;
    gvizSubgraphNeighborIterator it = gvizSubgraphNeighborIteratorCreate(&eg->subgraph, v);
    size_t u;
    while (gvizSubgraphNeighborIterate(&it, &u)) {
      if (n == cap) {
        cap *= 2;
        uint32_t *grown = realloc(col, cap * sizeof(uint32_t));
        if (!grown) {
          free(row), free(col), free(a), free(xy);
          return GVIZ_CUDA_ERR_ALLOC;
        }
        col = grown;
      }
      col[n++] = (uint32_t)u;
    }
  }
  row[V] = n;
  int rc = gvizCudaGripCreate(&a->h, V, row, col, device);
  free(row);
  free(col);
  if (rc) {
    free(a), free(xy);
    return rc;
  }
  gvizCudaGripSetStrictReductions(a->h, strictReductions);
  a->state = state;
  a->V = V;
  a->xy = xy;
  a->layer = (size_t)-1;
  if (gvizEmbeddedGraphAddAction(eg, "grip.refineRound", grip_gpu_action, NULL) < 0) {
    gvizCudaGripDestroy(a->h);
    free(a), free(xy);
    return GVIZ_CUDA_ERR_ALLOC;
  }
  a->next = g_grip;
  g_grip = a;
  return GVIZ_CUDA_OK;
}

/* the layer's filtration order and the state's k-nearest lists */
static int grip_push_layer(gripAttached *a) {
  gvizGRIPState *s = a->state;
  const size_t n = grip_active_count(s);
  uint32_t *act = malloc((n ? n : 1) * sizeof(uint32_t));
  uint64_t *off = malloc((n + 1) * sizeof(uint64_t));
  size_t total = 0;
  for (size_t i = 0; i < n; i++) total += s->dec[s->misFiltration[i]].knn.count;
  uint32_t *kv = malloc((total ? total : 1) * sizeof(uint32_t));
  uint32_t *kd = malloc((total ? total : 1) * sizeof(uint32_t));
  int rc = GVIZ_CUDA_OK;
  if (!act || !off || !kv || !kd) rc = GVIZ_CUDA_ERR_ALLOC;
  if (!rc) {
    size_t k = 0;
    for (size_t i = 0; i < n; i++) {
      const size_t v = s->misFiltration[i];
      const gvizArray *l = &s->dec[v].knn;
      act[i] = (uint32_t)v;
      off[i] = k;
      for (size_t j = 0; j < l->count; j++, k++) {
        const gvizFoundVertex *f = (const gvizFoundVertex *)gvizArrayAtIndex((gvizArray *)l, j);
        kv[k] = (uint32_t)f->v;
        kd[k] = (uint32_t)f->dist;
      }
    }
    off[n] = k;
    rc = gvizCudaGripSetLayer(a->h, s->currLayer, act, n, off, kv, kd);
  }
  free(act), free(off), free(kv), free(kd);
  if (!rc) {
    a->layer = s->currLayer;
    a->active = n;
    a->rounds = 0;
  }
  return rc;
}

void gvizCudaGripEmbedderRefineRound(gvizGRIPState *state) {
  gripAttached *a = grip_find(state);
  if (!a || state->layerCount == 0) return;
  gvizEmbeddedGraph *eg = (gvizEmbeddedGraph *)state;
  int rc = GVIZ_CUDA_OK;
  if (a->layer != state->currLayer || a->active != grip_active_count(state))
    rc = grip_push_layer(a);
  /* the embedding stays authoritative: positions go up and come back */
  for (size_t v = 0; v < a->V && !rc; v++) {
    const double *p = gvizEmbeddedGraphGetVPosition(eg, v);
    a->xy[2 * v] = p[0];
    a->xy[2 * v + 1] = p[1];
  }
  if (!rc) rc = gvizCudaGripSetPositions(a->h, a->xy);
  gvizCudaGripRoundStats st;
  if (!rc) rc = gvizCudaGripRefineRound(a->h, &st);
  if (!rc) rc = gvizCudaGripGetPositions(a->h, a->xy);
  if (rc) {
    a->lastError = rc;
    return;
  }
  for (size_t i = 0; i < a->active; i++) {
    const size_t v = state->misFiltration[i];
    double p[2] = {a->xy[2 * v], a->xy[2 * v + 1]};
    gvizEmbeddedGraphSetVPosition(eg, v, p);
  }
  state->lastRoundStats.maxDisplacement = st.maxDisplacement;
  state->lastRoundStats.meanDisplacement = st.meanDisplacement;
  state->lastRoundStats.meanForce = st.meanForce;
  if (state->statsEnabled) {
    gvizEmbeddedGraphStatAppend(eg, "grip.heat", st.meanHeat);
    gvizEmbeddedGraphStatAppend(eg, "grip.meanDisp", st.meanDisplacement);
    gvizEmbeddedGraphStatAppend(eg, "grip.maxDisp", st.maxDisplacement);
    gvizEmbeddedGraphStatAppend(eg, "grip.meanForce", st.meanForce);
  }
  state->currRound++;
  a->rounds++;
  a->lastError = 0;
}

void gvizCudaGripDetach(gvizGRIPState *state) {
  gripAttached **pp = &g_grip;
  while (*pp && (*pp)->state != state) pp = &(*pp)->next;
  gripAttached *a = *pp;
  if (!a) return;
  *pp = a->next;
  /* decorators of the layer the GPU worked on go back to the state */
  if (a->layer == state->currLayer && a->rounds > 0) {
    double *heat = malloc(a->V * sizeof(double)), *oc = malloc(a->V * sizeof(double));
    if (heat && oc && gvizCudaGripGetDecorators(a->h, heat, a->xy, oc) == GVIZ_CUDA_OK) {
      for (size_t i = 0; i < a->active; i++) {
        const size_t v = state->misFiltration[i];
        state->dec[v].heat = heat[v];
        state->dec[v].oldCos = oc[v];
        state->dec[v].disp[0] = a->xy[2 * v];
        state->dec[v].disp[1] = a->xy[2 * v + 1];
        gvizSetBit(state->dispCalculated, v);
      }
    }
    free(heat), free(oc);
  }
  gvizEmbeddedGraphAddAction((gvizEmbeddedGraph *)state, "grip.refineRound", grip_cpu_action,
                             NULL);
  gvizCudaGripDestroy(a->h);
  free(a->xy);
  free(a);
}

int gvizCudaGripEmbedderLastError(const gvizGRIPState *state) {
  const gripAttached *a = grip_find(state);
  return a ? a->lastError : GVIZ_CUDA_ERR_ARG;
}
