// rak_mtx.cpp -- Matrix Market (coordinate) graph ingest on the host, with the reference's reading
// rules (inc/mtx.hxx readMtxHeader :40-56, readMtxDoOmp :152-191, readMtxIfOmpW :251-260;
// inc/symmetrize.hxx symmetrizeOmpU :44-69), so SuiteSparse/SNAP-style inputs run through the
// library as the reference's driver reads them (main.cxx:118-119):
//   - banner "%%MatrixMarket matrix coordinate <field> <symmetry>"; other objects/formats give an
//     empty graph; "symmetric" and "skew-symmetric" store both directions of every entry;
//   - entries are 1-based "u v [w]"; weights are read only when asked, and a weight of 0 reads as 1
//     (the parallel reader's rule); unweighted graphs get weight 1;
//   - a repeated (u, v) keeps one edge, the weight of its last occurrence in the file;
//   - with symmetrize, every edge u->v whose reverse is missing gains v->u with the same weight;
//   - vertex ids become 0-based (u-1); n = max(rows, cols).
// Parsing runs on OpenMP threads over the file held in memory.
#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rak_lowmem.h"

namespace {

struct Threads {
  explicit Threads(int t) : saved(omp_get_max_threads()) { if (t > 0) omp_set_num_threads(t); }
  ~Threads() { omp_set_num_threads(saved); }
  int saved;
};

struct Entry {
  uint64_t key;   // u << 32 | v (0-based)
  uint64_t rank;  // position in reading order; ties keep the highest
  float w;
};

bool read_file(const char *path, std::string &buf) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz < 0) { std::fclose(f); return false; }
  buf.resize(size_t(sz));
  const size_t got = sz > 0 ? std::fread(&buf[0], 1, size_t(sz), f) : 0;
  std::fclose(f);
  return got == size_t(sz);
}

}  // namespace

extern "C" {

rak_status rak_read_mtx(const char *path, int weighted, int symmetrize, int threads, rak_host_csr *out) {
  if (!path || !out) return RAK_ERR_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  Threads th(threads);
  std::string text;
  if (!read_file(path, text)) return RAK_ERR_INVALID_ARGUMENT;
  // header: comment lines start with '%'; the banner starts with "%%"
  size_t pos = 0;
  std::string h1, h2, h4;
  std::string line;
  auto next_line = [&](std::string &l) {
    if (pos >= text.size()) return false;
    size_t e = text.find('\n', pos);
    if (e == std::string::npos) e = text.size();
    l.assign(text, pos, e - pos);
    pos = e + 1;
    return true;
  };
  bool have_size_line = false;
  while (next_line(line)) {
    if (line.rfind("%", 0) != 0) { have_size_line = true; break; }
    if (line.rfind("%%", 0) != 0) continue;
    char a[64] = {}, b[64] = {}, c[64] = {}, d[64] = {}, e[64] = {};
    std::sscanf(line.c_str(), "%63s %63s %63s %63s %63s", a, b, c, d, e);
    h1 = b;
    h2 = c;
    h4 = e;
  }
  out->offsets = static_cast<int64_t *>(std::calloc(1, 8));
  if (!out->offsets) return RAK_ERR_OUT_OF_MEMORY;
  if (!have_size_line || h1 != "matrix" || h2 != "coordinate") return RAK_OK;  // empty graph
  const bool symmetric = h4 == "symmetric" || h4 == "skew-symmetric";
  unsigned long long rows = 0, cols = 0, size = 0;
  if (std::sscanf(line.c_str(), "%llu %llu %llu", &rows, &cols, &size) < 2) return RAK_OK;
  const int64_t n = int64_t(std::max(rows, cols));
  if (n >= (int64_t(1) << 31)) { rak_host_csr_free(out); return RAK_ERR_INVALID_ARGUMENT; }
  // body lines
  std::vector<size_t> starts;
  starts.reserve(size_t(size) + 1);
  for (size_t p = pos; p < text.size();) {
    size_t e = text.find('\n', p);
    if (e == std::string::npos) e = text.size();
    if (e > p) starts.push_back(p);
    p = e + 1;
  }
  const int64_t L = int64_t(starts.size());
  std::vector<uint32_t> eu(static_cast<size_t>(L)), ev(static_cast<size_t>(L));
  std::vector<float> ew(static_cast<size_t>(L));
  std::vector<uint8_t> ok(static_cast<size_t>(L), uint8_t(0));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < L; ++i) {
    const char *s = text.c_str() + starts[size_t(i)];
    char *end = nullptr;
    const unsigned long long u = std::strtoull(s, &end, 10);
    if (end == s) continue;
    const char *s2 = end;
    const unsigned long long v = std::strtoull(s2, &end, 10);
    if (end == s2) continue;
    double w = 1;
    if (weighted) {
      const char *s3 = end;
      w = std::strtod(s3, &end);
      if (end == s3) w = 0;
      if (w == 0) w = 1;
    }
    if (u < 1 || v < 1 || int64_t(u) > n || int64_t(v) > n) continue;
    eu[size_t(i)] = uint32_t(u - 1);
    ev[size_t(i)] = uint32_t(v - 1);
    ew[size_t(i)] = float(w);
    ok[size_t(i)] = 1;
  }
  // directed entries in reading order (both directions for symmetric files)
  std::vector<Entry> es;
  es.reserve(size_t(L) * (symmetric ? 2 : 1));
  uint64_t rank = 0;
  for (int64_t i = 0; i < L; ++i) {
    if (!ok[size_t(i)]) continue;
    const uint64_t u = eu[size_t(i)], v = ev[size_t(i)];
    es.push_back({u << 32 | v, rank++, ew[size_t(i)]});
    if (symmetric) es.push_back({v << 32 | u, rank++, ew[size_t(i)]});
  }
  auto by_key_rank = [](const Entry &a, const Entry &b) { return a.key != b.key ? a.key < b.key : a.rank < b.rank; };
  std::sort(es.begin(), es.end(), by_key_rank);
  // a repeated pair keeps its last occurrence
  std::vector<Entry> uniq;
  uniq.reserve(es.size());
  for (size_t i = 0; i < es.size(); ++i)
    if (i + 1 == es.size() || es[i + 1].key != es[i].key) uniq.push_back(es[i]);
  es.clear();
  es.shrink_to_fit();
  if (symmetrize && !symmetric) {
    // reverse of every edge whose reverse is missing, with the edge's weight
    const size_t D = uniq.size();
    for (size_t i = 0; i < D; ++i) {
      const uint64_t u = uniq[i].key >> 32, v = uniq[i].key & 0xFFFFFFFFull;
      const uint64_t rk = v << 32 | u;
      const auto it = std::lower_bound(uniq.begin(), uniq.begin() + D, rk,
                                       [](const Entry &a, uint64_t k) { return a.key < k; });
      if (it == uniq.begin() + D || it->key != rk) uniq.push_back({rk, 0, uniq[i].w});
    }
    std::sort(uniq.begin(), uniq.end(), by_key_rank);
  }
  const int64_t m = int64_t(uniq.size());
  std::free(out->offsets);
  out->offsets = static_cast<int64_t *>(std::calloc(size_t(n + 1), 8));
  out->targets = static_cast<uint32_t *>(std::malloc(size_t(std::max<int64_t>(m, 1)) * 4));
  if (weighted) out->weights = static_cast<float *>(std::malloc(size_t(std::max<int64_t>(m, 1)) * 4));
  if (!out->offsets || !out->targets || (weighted && !out->weights)) {
    rak_host_csr_free(out);
    return RAK_ERR_OUT_OF_MEMORY;
  }
  for (int64_t i = 0; i < m; ++i) {
    out->offsets[(uniq[size_t(i)].key >> 32) + 1]++;
    out->targets[i] = uint32_t(uniq[size_t(i)].key & 0xFFFFFFFFull);
    if (weighted) out->weights[i] = uniq[size_t(i)].w;
  }
  for (int64_t u = 0; u < n; ++u) out->offsets[u + 1] += out->offsets[u];
  out->n = n;
  out->m = m;
  return RAK_OK;
}

}  // extern "C"
