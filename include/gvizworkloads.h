/* gvizworkloads.h -- seeded synthetic graphs (libgvizworkloads.so).
 *
 * A host-only C library kept apart from libgvizcuda, so that a process that
 * must not load the layout library (the CPU reference timing, for one) can
 * build the same inputs. Not part of the layout path itself: the reference
 * has fixture builders of its own (src/utils/graphs.c), two of which are
 * reproduced here edge for edge.
 */
#ifndef GVIZWORKLOADS_H
#define GVIZWORKLOADS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Ordered undirected edge lists. Each returns the edge count; pass NULL
 * buffers to query it first. */
/* build_rect_mesh (src/utils/graphs.c:285-316) */
size_t gvizGenGrid(size_t rows, size_t cols, uint32_t *ea, uint32_t *eb);
/* build_random_connected_graph (src/utils/graphs.c:598-639), same rand_r
 * stream, same edge order */
size_t gvizGenRandomConnected(size_t n, double density, unsigned seed,
                              uint32_t *ea, uint32_t *eb);
/* Barabasi-Albert: K_{m+1} seed, then each new vertex attaches m distinct
 * targets chosen proportionally to degree; 4n - 10 edges for m = 4 */
size_t gvizGenBarabasiAlbert(size_t n, uint32_t m, uint64_t seed,
                             uint32_t *ea, uint32_t *eb);
/* Erdos-Renyi G(n, m): m distinct non-loop edges */
size_t gvizGenErdosRenyi(size_t n, size_t m, uint64_t seed, uint32_t *ea,
                         uint32_t *eb);
/* R-MAT with (a, b, c, 1-a-b-c): `draws` edge draws, self-loops dropped,
 * duplicates (either orientation) removed, first occurrence kept */
size_t gvizGenRmat(uint32_t scale, size_t draws, double a, double b,
                   double c, uint64_t seed, uint32_t *ea, uint32_t *eb);

#ifdef __cplusplus
}
#endif

#endif /* GVIZWORKLOADS_H */
