/*
 * gvizCudaGripEmbedder.h -- gviz-side glue that moves an existing
 * gvizGRIPState's refinement rounds onto libgvizcuda (gvizCudaGrip*).
 *
 * Compiled inside gviz (it includes gviz's own headers). After
 * gvizGRIPEmbedderInit, gvizCudaGripAttach copies the subgraph's structure
 * to the GPU and re-registers the "grip.refineRound" action
 * (src/embedders/gvizGRIPEmbedder.c:158-166, registered at :291-293), so
 * front-ends that invoke it by name refine on the GPU unchanged; registering
 * the same name replaces the handler (src/embedders/gvizEmbeddedGraph.c:227-232).
 *
 * Every round keeps gvizGRIPEmbedderRefineRound's observable contract
 * (:1289-1334): the active vertices' positions are read from and written back
 * to the embedding, lastRoundStats is set, currRound advances and the four
 * "grip.*" stat series get one sample each when stats are on. GRIP's MIS
 * filtration, placement and k-nearest search stay in gviz: when the layer
 * changes (gvizGRIPEmbedderBegin / NextStage, or the "grip.nextStage"
 * action) the next GPU round takes the layer's filtration order and the
 * state's own k-nearest lists. Decorators (heat, displacement, cosine) live
 * on the GPU while attached and are written back to the state at detach.
 */
#ifndef GVIZ_CUDA_GRIP_EMBEDDER_H
#define GVIZ_CUDA_GRIP_EMBEDDER_H

#include "embedders/gvizGRIPEmbedder.h"
#include "gvizcuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Attaches the GPU rounds to an initialised 2-D GRIP state and takes over the
 * "grip.refineRound" action. strictReductions = 1: every round bit-identical
 * to the reference's serial round. Returns 0, -2 (dimension != 2) or another
 * GVIZ_CUDA_ERR_* code. */
int gvizCudaGripAttach(gvizGRIPState *state, int32_t device, int32_t strictReductions);

/* gvizGRIPEmbedderRefineRound (src/embedders/gvizGRIPEmbedder.c:1289-1334)
 * on the GPU; a no-op before gvizGRIPEmbedderBegin. */
void gvizCudaGripEmbedderRefineRound(gvizGRIPState *state);

/* Writes the decorators back, gives "grip.refineRound" back to the CPU round
 * and frees the GPU handle. */
void gvizCudaGripDetach(gvizGRIPState *state);

/* Last GVIZ_CUDA_ERR_* seen for this state (0 when none). */
int gvizCudaGripEmbedderLastError(const gvizGRIPState *state);

#ifdef __cplusplus
}
#endif

#endif
