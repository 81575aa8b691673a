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

#include <string>
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

// ---- GEXF (src/utils/graphLoader.c:186-800): the tag scanner's rules ----
// A tag is its name followed by a blank, '/' or '>'; it ends at the first
// '>' after it; an attribute is the first `name="` (else `name='`) inside
// the tag, its value up to the matching quote and shorter than the
// loader's buffer. Kept alike so that a file loads, or fails, the same way.

bool gexf_tag_char(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '/' || c == '>';
}

const char *gexf_tag(const char *from, const char *name) {
  const size_t n = strlen(name);
  for (const char *p = from; (p = strstr(p, name)) != nullptr; p += n)
    if (gexf_tag_char(p[n])) return p;
  return nullptr;
}

// first occurrence of needle wholly inside [hay, end)
const char *gexf_find(const char *hay, const char *end, const char *needle) {
  const size_t n = strlen(needle);
  if (n == 0 || end < hay || n > (size_t)(end - hay)) return nullptr;
  for (const char *p = hay; p + n <= end; p++)
    if (memcmp(p, needle, n) == 0) return p;
  return nullptr;
}

const char *gexf_tag_in(const char *from, const char *end, const char *name) {
  const size_t n = strlen(name);
  for (const char *p = from; p < end;) {
    const char *f = gexf_find(p, end, name);
    if (!f) return nullptr;
    if (f + n <= end && gexf_tag_char(f[n])) return f;
    p = f + n;
  }
  return nullptr;
}

// 0 with the value in out, or -1 (absent, unterminated, or cap or longer)
int gexf_attr(const char *ts, const char *te, const char *name, std::string &out, size_t cap) {
  std::string pat = std::string(name) + "=\"";
  char quote = '"';
  const char *p = gexf_find(ts, te, pat.c_str());
  if (!p) {
    pat = std::string(name) + "='";
    quote = '\'';
    p = gexf_find(ts, te, pat.c_str());
  }
  if (!p) return -1;
  p += pat.size();
  const char *q = static_cast<const char *>(memchr(p, quote, (size_t)(te - p)));
  if (!q || (size_t)(q - p) >= cap) return -1;
  out.assign(p, q);
  return 0;
}

// The checks of the attribute-type table (node attributes need an id);
// the types themselves only shape gviz's per-vertex JSON, which the layout
// does not use.
int gexf_check_attribute_types(const char *buf) {
  std::string v;
  for (const char *p = buf, *ts; (ts = gexf_tag(p, "<attributes")) != nullptr;) {
    const char *te = strchr(ts, '>');
    if (!te) return -1;
    const bool edgeClass = gexf_attr(ts, te, "class", v, 32) == 0 && v == "edge";
    const char *body = te + 1;
    const char *bodyEnd = strstr(body, "</attributes>");
    if (!bodyEnd) return -1;
    if (!edgeClass) {
      for (const char *ap = body, *at; (at = gexf_tag_in(ap, bodyEnd, "<attribute")) != nullptr;) {
        const char *ate = static_cast<const char *>(memchr(at, '>', (size_t)(bodyEnd - at)));
        if (!ate || gexf_attr(at, ate, "id", v, 256) < 0) return -1;
        ap = ate + 1;
      }
    }
    p = bodyEnd + strlen("</attributes>");
  }
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

int gvizCudaLoadGexfFile(const char *path, gvizCudaCsr *out) {
  if (!path || !out) return -1;
  memset(out, 0, sizeof(*out));
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  std::string text;
  if (fseek(f, 0, SEEK_END) != 0) {
    fclose(f);
    return -1;
  }
  const long size = ftell(f);
  if (size < 0 || fseek(f, 0, SEEK_SET) != 0) {
    fclose(f);
    return -1;
  }
  try {
    text.resize((size_t)size);
    text.resize(fread(&text[0], 1, (size_t)size, f));
  } catch (...) {
    fclose(f);
    return -1;
  }
  fclose(f);
  const char *buf = text.c_str();  // scanned as a C string, as gviz does
  try {
    size_t nodeTags = 0;
    for (const char *p = buf; (p = gexf_tag(p, "<node")) != nullptr; p += 5) nodeTags++;
    if (nodeTags == 0 || nodeTags >= 0xffffffffull) return -1;
    if (gexf_check_attribute_types(buf) < 0) return -1;
    // vertices in tag order; an id names the first vertex that carried it
    std::unordered_map<std::string, uint32_t> ids;
    ids.reserve(nodeTags * 2);
    uint32_t V = 0;
    std::string id, v1, v2;
    for (const char *p = buf, *ts; (ts = gexf_tag(p, "<node")) != nullptr;) {
      const char *te = strchr(ts, '>');
      if (!te || gexf_attr(ts, te, "id", id, 256) < 0) return -1;
      const char *next = te + 1;
      if (!(te > ts && te[-1] == '/')) {
        const char *close = strstr(te + 1, "</node>");
        if (!close) return -1;
        // <attvalue for|id="..." value="..."> entries must parse
        for (const char *ap = te + 1, *at; (at = gexf_tag_in(ap, close, "<attvalue")) != nullptr;) {
          const char *ate = static_cast<const char *>(memchr(at, '>', (size_t)(close - at)));
          if (!ate) return -1;
          if ((gexf_attr(at, ate, "for", v1, 256) < 0 && gexf_attr(at, ate, "id", v1, 256) < 0) ||
              gexf_attr(at, ate, "value", v2, 512) < 0)
            return -1;
          ap = ate + 1;
        }
        next = close + strlen("</node>");
      }
      ids.emplace(id, V);
      V++;
      p = next;
    }
    // undirected edges in tag order; both ends must name vertices
    std::vector<uint32_t> ea, eb;
    for (const char *p = buf, *ts; (ts = gexf_tag(p, "<edge")) != nullptr;) {
      const char *te = strchr(ts, '>');
      if (!te || gexf_attr(ts, te, "source", v1, 256) < 0 ||
          gexf_attr(ts, te, "target", v2, 256) < 0)
        return -1;
      const auto a = ids.find(v1), b = ids.find(v2);
      if (a == ids.end() || b == ids.end()) return -1;
      ea.push_back(a->second);
      eb.push_back(b->second);
      p = te + 1;
    }
    return edges_to_csr(V, ea, eb, 0, out);
  } catch (...) {
    memset(out, 0, sizeof(*out));
    return -1;
  }
}

}  // extern "C"
