/*
 * gvizCudaForceEmbedder.h -- gviz-side glue that moves an existing
 * gvizForceEmbedderState's steps onto libgvizcuda.
 *
 * Compiled inside gviz (it includes gviz's own headers). After
 * gvizForceEmbedderInit (+ Configure*), gvizCudaForceAttach copies the
 * subgraph's structure to the GPU and re-registers the "forceEmbedder.step"
 * action, so front-ends that invoke the action by name
 * (src/embedders/gvizEmbeddedGraph.c:283-293) step on the GPU unchanged;
 * registering the same name replaces the handler
 * (src/embedders/gvizEmbeddedGraph.c:227-232).
 *
 * Every step keeps the reference's observable contract
 * (src/embedders/gvizForceEmbedder.c:445-495): positions are read from and
 * written back to the embedding, iteration and lastMaxDisplacement advance,
 * globalSpeed / speedEfficiency are updated and the five stat series get one
 * sample each. Configuration fields (theta, preventOverlap, ...) are re-read
 * every step, so the "forceEmbedder.toggleOverlapPrevention" action keeps
 * working. A Begin (iteration back to 0) or interleaved CPU steps are detected
 * and the FA2 history is re-uploaded from the state.
 */
#ifndef GVIZ_CUDA_FORCE_EMBEDDER_H
#define GVIZ_CUDA_FORCE_EMBEDDER_H

#include "embedders/gvizForceEmbedder.h"
#include "gvizcuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gvizCudaOptions {
  int32_t device;      /* CUDA device ordinal */
  int32_t precision;   /* GVIZ_CUDA_FP32 (fast) or GVIZ_CUDA_FP64 (reference
                          operation order) */
  int32_t syncScratch; /* 1: after every step also copy disp, structForce,
                          |att|, |rep|, swing, traction and appliedDisp into
                          the state's arrays (full drop-in); 0: positions,
                          speed and stats only */
  int32_t strictReductions; /* 1: global sums in vertex order */
} gvizCudaOptions;

/* Attaches the GPU path to an initialised embedder (after
 * gvizForceEmbedderInit, src/embedders/gvizForceEmbedder.c:219-325) and
 * takes over the "forceEmbedder.step" action. Returns 0, -1 (allocation),
 * -2 (dimension != 2) or another GVIZ_CUDA_ERR_* code. */
int gvizCudaForceAttach(gvizForceEmbedderState *state,
                        const gvizCudaOptions *options);

/* gvizForceEmbedderStep (src/embedders/gvizForceEmbedder.c:445-495) on the
 * GPU. Returns maxDisp, or a negative GVIZ_CUDA_ERR_* code. */
double gvizCudaForceEmbedderStep(gvizForceEmbedderState *state);

/* gvizForceEmbedderRun (src/embedders/gvizForceEmbedder.c:497-510) with the
 * loop resident on the GPU; -1 if Begin has not been called. */
int gvizCudaForceEmbedderRun(gvizForceEmbedderState *state, size_t maxIters,
                             double epsilon);

/* Gives the step back to the CPU implementation and frees the GPU handle. */
void gvizCudaForceDetach(gvizForceEmbedderState *state);

/* Last GVIZ_CUDA_ERR_* seen for this state (0 when none); the action
 * handler cannot return one. */
int gvizCudaForceEmbedderLastError(const gvizForceEmbedderState *state);

/* The library handle attached to this state (NULL when none), for options
 * the embedder has no field for: the learned far field
 * (gvizCudaForceSetFarFieldModel, then farField, farCellGroups,
 * farHubTargets, ... through gvizCudaForceGetParams / SetParams). Steps
 * through the action keep those options; every other field is re-read from
 * the state before each step. The handle stays owned by the attachment. */
gvizCudaForce *gvizCudaForceEmbedderHandle(const gvizForceEmbedderState *state);

/* gvizForceEmbedderRun (src/embedders/gvizForceEmbedder.c:497-510) for n
 * independent begun embedders at once, all laid out by one GPU handle (one
 * quadtree per graph in one forest, per-graph FA2 speed, per-graph
 * convergence), then written back to each state like n separate Runs:
 * positions, iteration, lastMaxDisplacement, globalSpeed, speedEfficiency,
 * the five stat series (each graph's latest 4096 rows) and, with
 * options->syncScratch, the per-vertex arrays. The embedders need not be
 * attached. They must share the force model and configuration (theta,
 * edgeLength, ...); otherwise GVIZ_CUDA_ERR_ARG. rounds[n] (may be NULL)
 * receives each graph's round count. Returns 0, -1 if one has not begun, or
 * a negative GVIZ_CUDA_ERR_* code. */
int gvizCudaForceEmbedderRunBatch(gvizForceEmbedderState **states, size_t n,
                                  size_t maxIters, double epsilon,
                                  const gvizCudaOptions *options, uint64_t *rounds);

#ifdef __cplusplus
}
#endif

#endif
