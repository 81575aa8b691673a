// loaders.cpp -- graph files straight to CSR (host code).
//
// gviz loads a file into its adjacency-list graph (per-vertex growable
// arrays, src/utils/graphLoader.c) and the layout then walks those lists.
// These loaders produce the layout's CSR directly, with the same vertex
// numbering and the same neighbour order as gviz's loaders followed by its
// subgraph neighbour iterator, so a file laid out here and in gviz gives the
// same graph. Errors follow gviz's loaders: -1 on I/O, parse or allocation
// failure, with the output zeroed.
#include <errno.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "gvizcuda.h"

namespace {

// One line at a time, any length (getline semantics).
struct LineReader {
  FILE *f = nullptr;
  char *buf = nullptr;
  size_t cap = 0;
  explicit LineReader(const char *path) : f(fopen(path, "r")) {}
  ~LineReader() {
    free(buf);
    if (f) fclose(f);
  }
  const char *next() { return getline(&buf, &cap, f) == -1 ? nullptr : buf; }
};

// The .edges line rule (src/utils/graphLoader.c:15-36): skip blanks; an
// empty line or a '%' comment is no edge (0); two base-10 integers read by
// strtoll are an edge (1); anything else is an error (-1). Further columns
// (a weight) are ignored.
int parse_edge_line(const char *line, long long *u, long long *v) {
  while (*line == ' ' || *line == '\t') line++;
  if (*line == '\0' || *line == '\n' || *line == '\r' || *line == '%') return 0;
  char *end = nullptr;
  const long long a = strtoll(line, &end, 10);
  if (end == line) return -1;
  line = end;
  while (*line == ' ' || *line == '\t') line++;
  const long long b = strtoll(line, &end, 10);
  if (end == line) return -1;
  *u = a;
  *v = b;
  return 1;
}

// CSR of an edge list added in order with gvizGraphAddEdge semantics
// (src/ds/gvizGraph.c:163-172): `from` gets `to`; undirected graphs also
// give `from` to `to` (a self-loop appears twice). Neighbour order is
// insertion order.
int edges_to_csr(size_t V, const std::vector<uint32_t> &ea, const std::vector<uint32_t> &eb,
                 int directed, gvizCudaCsr *out) {
  std::vector<uint64_t> cnt(V + 1, 0);
  for (size_t e = 0; e < ea.size(); e++) {
    cnt[ea[e]]++;
    if (!directed) cnt[eb[e]]++;
  }
  uint64_t *row = (uint64_t *)malloc(sizeof(uint64_t) * (V + 1));
  if (!row) return -1;
  row[0] = 0;
  for (size_t v = 0; v < V; v++) row[v + 1] = row[v] + cnt[v];
  const uint64_t entries = row[V];
  uint32_t *col = (uint32_t *)malloc(sizeof(uint32_t) * (entries ? entries : 1));
  if (!col) {
    free(row);
    return -1;
  }
  std::vector<uint64_t> cur(row, row + V);
  for (size_t e = 0; e < ea.size(); e++) {
    col[cur[ea[e]]++] = eb[e];
    if (!directed) col[cur[eb[e]]++] = ea[e];
  }
  out->vertexCount = V;
  out->entryCount = entries;
  out->rowOffsets = row;
  out->neighbors = col;
  out->directed = directed;
  return 0;
}

}  // namespace

extern "C" {

void gvizCudaCsrFree(gvizCudaCsr *csr) {
  if (!csr) return;
  free(csr->rowOffsets);
  free(csr->neighbors);
  free(csr->externalIds);
  memset(csr, 0, sizeof(*csr));
}

int gvizCudaLoadEdgesFile(const char *path, int directed, int skipHeader, gvizCudaCsr *out) {
  if (!path || !out) return -1;
  memset(out, 0, sizeof(*out));
  LineReader in(path);
  if (!in.f) return -1;
  // internal ids in order of first appearance (u, then v, line by line),
  // as gviz's loader assigns them (src/utils/graphLoader.c:112-126)
  std::unordered_map<long long, uint32_t> id;
  std::vector<long long> ext;
  std::vector<uint32_t> ea, eb;
  bool skip = skipHeader != 0;
  try {
    for (const char *line; (line = in.next()) != nullptr;) {
      long long u = 0, v = 0;
      const int parsed = parse_edge_line(line, &u, &v);
      if (parsed < 0) return -1;
      if (parsed == 0) continue;
      if (skip) {
        skip = false;
        continue;
      }
      if (u < 0 || v < 0) return -1;
      uint32_t iu, iv;
      for (int k = 0; k < 2; k++) {
        const long long x = k ? v : u;
        auto it = id.find(x);
        uint32_t i;
        if (it == id.end()) {
          if (ext.size() >= 0xffffffffull) return -1;  // 32-bit CSR indices
          i = (uint32_t)ext.size();
          id.emplace(x, i);
          ext.push_back(x);
        } else {
          i = it->second;
        }
        (k ? iv : iu) = i;
      }
      ea.push_back(iu);
      eb.push_back(iv);
    }
  } catch (...) {  // std::bad_alloc
    return -1;
  }
  if (ext.empty()) return -1;  // no edge at all: gviz fails too
  if (edges_to_csr(ext.size(), ea, eb, directed, out) != 0) return -1;
  out->externalIds = (int64_t *)malloc(sizeof(int64_t) * ext.size());
  if (!out->externalIds) {
    gvizCudaCsrFree(out);
    return -1;
  }
  for (size_t i = 0; i < ext.size(); i++) out->externalIds[i] = ext[i];
  return 0;
}

int gvizCudaLoadObjFile(const char *path, gvizCudaCsr *out) {
  if (!path || !out) return -1;
  memset(out, 0, sizeof(*out));
  LineReader in(path);
  if (!in.f) return -1;
  size_t V = 0;
  std::vector<uint32_t> ea, eb;
  std::unordered_set<uint64_t> seen;  // undirected edges (a < b) already added
  std::vector<size_t> face;
  try {
    for (const char *line; (line = in.next()) != nullptr;) {
      const char *p = line;
      while (*p == ' ' || *p == '\t') p++;
      if (*p == '\0' || *p == '\n' || *p == '\r' || *p == '#') continue;
      if (p[0] == 'v' && (p[1] == ' ' || p[1] == '\t')) {
        if (V >= 0xffffffffull) return -1;
        V++;
        continue;
      }
      if (!(p[0] == 'f' && (p[1] == ' ' || p[1] == '\t'))) continue;
      // a face: corner indices (1-based, or negative = relative to the
      // vertices so far), texture/normal parts after '/' ignored
      // (src/utils/graphLoader.c:827-917)
      face.clear();
      for (p += 2; *p;) {
        while (*p == ' ' || *p == '\t') p++;
        if (*p == '\0' || *p == '\n' || *p == '\r') break;
        char *end = nullptr;
        const long idx = strtol(p, &end, 10);
        if (end == p || idx == 0) return -1;
        size_t corner;
        if (idx > 0) {
          if ((size_t)idx > V) return -1;
          corner = (size_t)idx - 1;
        } else {
          if ((size_t)(-idx) > V) return -1;
          corner = V - (size_t)(-idx);
        }
        face.push_back(corner);
        while (*p && *p != ' ' && *p != '\t' && *p != '\n' && *p != '\r') p++;
      }
      if (face.size() < 2) continue;
      // consecutive corners and the closing edge, no self-loops, no repeats
      for (size_t i = 0; i < face.size(); i++) {
        size_t a = face[i], b = face[(i + 1) % face.size()];
        if (a == b) continue;
        if (a > b) std::swap(a, b);
        if (!seen.insert(((uint64_t)a << 32) | (uint64_t)b).second) continue;
        ea.push_back((uint32_t)a);
        eb.push_back((uint32_t)b);
      }
    }
  } catch (...) {
    return -1;
  }
  if (V == 0) return -1;
  return edges_to_csr(V, ea, eb, 0, out) == 0 ? 0 : -1;
}

}  // extern "C"
