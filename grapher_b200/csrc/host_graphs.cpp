// host_graphs.cpp -- CSR construction, the initial placement and GRIP's
// k-nearest search, host-side C++ behind the C ABI (include/gvizcuda.h).
// The synthetic workload generators live in their own library
// (workloads.cpp, include/gvizworkloads.h).
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "gvizcuda.h"


extern "C" {

int gvizCudaEdgesToCsr(size_t V, const uint32_t *ea, const uint32_t *eb,
                       size_t E, uint64_t *rowOffsets, uint32_t *neighbors) {
  if (!rowOffsets || (E && (!ea || !eb || !neighbors))) return GVIZ_CUDA_ERR_ARG;
  std::vector<uint64_t> cnt(V + 1, 0);
  for (size_t e = 0; e < E; e++) {
    if (ea[e] >= V || eb[e] >= V) return GVIZ_CUDA_ERR_ARG;
    cnt[ea[e]]++;
    cnt[eb[e]]++;
  }
  rowOffsets[0] = 0;
  for (size_t v = 0; v < V; v++) rowOffsets[v + 1] = rowOffsets[v] + cnt[v];
  std::vector<uint64_t> cur(rowOffsets, rowOffsets + V);
  for (size_t e = 0; e < E; e++) {
    neighbors[cur[ea[e]]++] = eb[e];
    neighbors[cur[eb[e]]++] = ea[e];
  }
  return GVIZ_CUDA_OK;
}

void gvizCudaRandomizePositions(double *xy, size_t V, double boxExtent,
                                unsigned seed) {
  if (!xy) return;
  if (seed == 0) seed = (unsigned)time(NULL);
  for (size_t i = 0; i < V; i++)
    for (int d = 0; d < 2; d++) {
      double unit = (double)rand_r(&seed) / ((double)RAND_MAX + 1.0);
      xy[2 * i + d] = boxExtent * (2.0 * unit - 1.0);
    }
}

// GRIP's k-nearest search (gvizSearchKNearestScratch,
// src/algorithms/search/gvizKNearest.c:244-306): a breadth-first search from
// each source over the whole graph, neighbours in CSR order, each vertex
// reached for the first time recorded with its depth when it is visible,
// until k are recorded. Sources run on all host threads, each with its own
// visit stamps; the result depends only on the inputs. Writes source i's
// list at offsets[i] (the lists packed in source order; vertices and
// distances need room for sourceCount * k entries) and returns the total.
int64_t gvizCudaGripKNearest(size_t vertexCount, const uint64_t *rowOffsets,
                             const uint32_t *neighbors, const uint32_t *sources,
                             size_t sourceCount, const uint8_t *visible, uint32_t k,
                             uint64_t *offsets, uint32_t *vertices, uint32_t *distances) {
  if (!rowOffsets || (sourceCount && (!sources || !offsets)) ||
      (sourceCount && k && (!vertices || !distances)))
    return GVIZ_CUDA_ERR_ARG;
  for (size_t i = 0; i < sourceCount; i++)
    if (sources[i] >= vertexCount) return GVIZ_CUDA_ERR_ARG;
  std::vector<uint32_t> count(sourceCount, 0);
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  if ((size_t)nt > sourceCount) nt = (unsigned)(sourceCount ? sourceCount : 1);
  auto work = [&](unsigned t) {
    std::vector<uint32_t> stamp(vertexCount, 0);
    std::vector<uint32_t> qv, qd;
    uint32_t epoch = 0;
    for (size_t i = t; i < sourceCount; i += nt) {
      const uint32_t src = sources[i];
      uint32_t *outV = vertices + i * (size_t)k;
      uint32_t *outD = distances + i * (size_t)k;
      uint32_t c = 0;
      if (k) {
        if (++epoch == 0) {
          std::fill(stamp.begin(), stamp.end(), 0u);
          epoch = 1;
        }
        qv.assign(1, src);
        qd.assign(1, 0);
        stamp[src] = epoch;
        for (size_t head = 0; head < qv.size() && c < k; head++) {
          const uint32_t u = qv[head], du = qd[head];
          for (uint64_t j = rowOffsets[u]; j < rowOffsets[u + 1]; j++) {
            const uint32_t w = neighbors[j];
            if (stamp[w] == epoch) continue;
            stamp[w] = epoch;
            if (!visible || visible[w]) {
              outV[c] = w;
              outD[c] = du + 1;
              if (++c >= k) break;
            }
            qv.push_back(w);
            qd.push_back(du + 1);
          }
        }
      }
      count[i] = c;
    }
  };
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < nt; t++) pool.emplace_back(work, t);
  work(0);
  for (auto &th : pool) th.join();
  // pack the lists in source order (each moves left or stays)
  uint64_t o = 0;
  for (size_t i = 0; i < sourceCount; i++) {
    offsets[i] = o;
    const uint32_t c = count[i];
    if (o != i * (uint64_t)k) {
      memmove(vertices + o, vertices + i * (size_t)k, c * sizeof(uint32_t));
      memmove(distances + o, distances + i * (size_t)k, c * sizeof(uint32_t));
    }
    o += c;
  }
  if (sourceCount) offsets[sourceCount] = o;
  return (int64_t)o;
}

}  // extern "C"
