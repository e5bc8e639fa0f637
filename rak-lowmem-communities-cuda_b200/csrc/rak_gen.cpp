// rak_gen.cpp -- deterministic synthetic graphs on the host (OpenMP): symmetric R-MAT, planted
// partition SBM and a perturbed 2D lattice. These stand in for the SuiteSparse/SNAP inputs of the
// reference's experiments (main.sh:42-56), which are not available here. Every random choice is a
// counter-based hash of (seed, stream, index), so results do not depend on the thread count.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "rak_hash.hpp"
#include "rak_lowmem.h"

namespace {

using rak::rand64;
using rak::unit24;

enum : uint64_t { STREAM_RMAT = 1, STREAM_WEIGHT = 2, STREAM_SBM = 3, STREAM_LATTICE = 4 };

struct Threads {
  explicit Threads(int t) : saved(omp_get_max_threads()) { if (t > 0) omp_set_num_threads(t); }
  ~Threads() { omp_set_num_threads(saved); }
  int saved;
};

// Builds a symmetric CSR with sorted, duplicate-free adjacency and no self-loops from samples
// gen(i, u, v) -> keep?, i in [0, samples). Both directions of every kept sample are stored.
template <class Gen>
rak_status build_symmetric(int64_t n, int64_t samples, Gen gen, rak_host_csr *out) {
  std::vector<uint32_t> cnt(size_t(n) + 1, 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < samples; ++i) {
    uint32_t u, v;
    if (!gen(i, u, v) || u == v) continue;
    __atomic_fetch_add(&cnt[u], 1u, __ATOMIC_RELAXED);
    __atomic_fetch_add(&cnt[v], 1u, __ATOMIC_RELAXED);
  }
  std::vector<int64_t> off(size_t(n) + 1, 0);
  for (int64_t u = 0; u < n; ++u) off[u + 1] = off[u] + cnt[u];
  const int64_t raw = off[n];
  uint32_t *tmp = static_cast<uint32_t *>(std::malloc(size_t(std::max<int64_t>(raw, 1)) * 4));
  if (!tmp) return RAK_ERR_OUT_OF_MEMORY;
  std::vector<int64_t> cur(off.begin(), off.end() - 1);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < samples; ++i) {
    uint32_t u, v;
    if (!gen(i, u, v) || u == v) continue;
    tmp[__atomic_fetch_add(&cur[u], int64_t(1), __ATOMIC_RELAXED)] = v;
    tmp[__atomic_fetch_add(&cur[v], int64_t(1), __ATOMIC_RELAXED)] = u;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < n; ++u) {
    uint32_t *b = tmp + off[u], *e = tmp + off[u + 1];
    std::sort(b, e);
    cnt[u] = uint32_t(std::unique(b, e) - b);
  }
  out->n = n;
  out->offsets = static_cast<int64_t *>(std::malloc(size_t(n + 1) * 8));
  if (!out->offsets) { std::free(tmp); return RAK_ERR_OUT_OF_MEMORY; }
  out->offsets[0] = 0;
  for (int64_t u = 0; u < n; ++u) out->offsets[u + 1] = out->offsets[u] + cnt[u];
  out->m = out->offsets[n];
  out->targets = static_cast<uint32_t *>(std::malloc(size_t(std::max<int64_t>(out->m, 1)) * 4));
  if (!out->targets) { std::free(tmp); std::free(out->offsets); out->offsets = nullptr; return RAK_ERR_OUT_OF_MEMORY; }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < n; ++u)
    std::memcpy(out->targets + out->offsets[u], tmp + off[u], size_t(cnt[u]) * 4);
  std::free(tmp);
  return RAK_OK;
}

// Symmetric weights: one value in [lo, hi) per undirected pair, from the pair's hash.
rak_status fill_weights(rak_host_csr *g, uint64_t seed, float lo, float hi) {
  g->weights = static_cast<float *>(std::malloc(size_t(std::max<int64_t>(g->m, 1)) * 4));
  if (!g->weights) return RAK_ERR_OUT_OF_MEMORY;
  const float span = hi - lo;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < g->n; ++u)
    for (int64_t e = g->offsets[u]; e < g->offsets[u + 1]; ++e) {
      uint64_t a = uint64_t(u), b = g->targets[e];
      uint64_t key = a < b ? (a << 32 | b) : (b << 32 | a);
      float t = span * unit24(rand64(seed, STREAM_WEIGHT, key));
      g->weights[e] = lo + t;
    }
  return RAK_OK;
}

void clear(rak_host_csr *g) { std::memset(g, 0, sizeof(*g)); }

// Uniform integer in [0, n) from 32 random bits (n < 2^32).
inline uint32_t below(uint64_t h, uint64_t n) { return uint32_t(((h >> 32) * n) >> 32); }

}  // namespace

extern "C" {

rak_status rak_gen_rmat(int scale, double edge_factor, double a, double b, double c, uint64_t seed,
                        float w_lo, float w_hi, int threads, rak_host_csr *out) {
  if (!out || scale < 1 || scale > 31 || !(edge_factor > 0) || a < 0 || b < 0 || c < 0 ||
      a + b + c > 1.0 || w_hi < w_lo)
    return RAK_ERR_INVALID_ARGUMENT;
  clear(out);
  Threads th(threads);
  const int64_t n = int64_t(1) << scale;
  const int64_t samples = int64_t(std::llround(double(n) * edge_factor));
  const uint32_t tA = uint32_t(std::lround(a * 65536.0));
  const uint32_t tAB = uint32_t(std::lround((a + b) * 65536.0));
  const uint32_t tABC = uint32_t(std::lround((a + b + c) * 65536.0));
  // Each level takes 16 random bits; quadrant (0,0) with probability a, (0,1) b, (1,0) c, (1,1) d.
  auto gen = [=](int64_t i, uint32_t &u, uint32_t &v) {
    uint32_t uu = 0, vv = 0;
    uint64_t h = 0;
    for (int L = 0; L < scale; ++L) {
      if ((L & 3) == 0) h = rand64(seed, STREAM_RMAT, uint64_t(i) * 8 + uint64_t(L >> 2));
      uint32_t r = uint32_t(h >> (16 * (L & 3))) & 0xFFFFu;
      uint32_t ub = r >= tAB;
      uint32_t vb = (r >= tA && r < tAB) || r >= tABC;
      uu = (uu << 1) | ub;
      vv = (vv << 1) | vb;
    }
    u = uu; v = vv;
    return true;
  };
  rak_status st = build_symmetric(n, samples, gen, out);
  if (st != RAK_OK) return st;
  if (!(w_lo == 1.0f && w_hi == 1.0f)) {
    st = fill_weights(out, seed, w_lo, w_hi);
    if (st != RAK_OK) { rak_host_csr_free(out); return st; }
  }
  return RAK_OK;
}

rak_status rak_gen_sbm(int64_t n, int64_t k, double avg_degree, double in_out_ratio, uint64_t seed,
                       int threads, rak_host_csr *out) {
  if (!out || n < 2 || n >= (int64_t(1) << 31) || k < 1 || k > n || !(avg_degree > 0) || !(in_out_ratio > 0))
    return RAK_ERR_INVALID_ARGUMENT;
  clear(out);
  Threads th(threads);
  auto start = [=](int64_t blk) { return (blk * n + k - 1) / k; };  // block of u is floor(u*k/n)
  const double s = double(n) / double(k);
  // Fraction of a vertex's expected degree that falls inside its own block when
  // p_in/p_out = in_out_ratio: r(s-1) / (r(s-1) + (n-s)).
  const double fin = k == 1 ? 1.0 : in_out_ratio * (s - 1) / (in_out_ratio * (s - 1) + (double(n) - s));
  const uint32_t fin24 = uint32_t(std::lround(fin * 16777216.0));
  const int64_t samples = int64_t(std::llround(double(n) * avg_degree / 2.0));
  auto gen = [=](int64_t i, uint32_t &u, uint32_t &v) {
    uint64_t h0 = rand64(seed, STREAM_SBM, uint64_t(i) * 3);
    uint64_t h1 = rand64(seed, STREAM_SBM, uint64_t(i) * 3 + 1);
    uint64_t h2 = rand64(seed, STREAM_SBM, uint64_t(i) * 3 + 2);
    u = below(h0, uint64_t(n));
    int64_t blk = int64_t(u) * k / n, lo = start(blk), hi = start(blk + 1);
    if (uint32_t(h1 >> 40) < fin24 || hi - lo == n) {
      v = uint32_t(lo) + below(h2, uint64_t(hi - lo));
    } else {
      uint32_t r = below(h2, uint64_t(n - (hi - lo)));
      v = r < uint32_t(lo) ? r : r + uint32_t(hi - lo);
    }
    return true;
  };
  rak_status st = build_symmetric(n, samples, gen, out);
  if (st != RAK_OK) return st;
  out->truth = static_cast<uint32_t *>(std::malloc(size_t(n) * 4));
  if (!out->truth) { rak_host_csr_free(out); return RAK_ERR_OUT_OF_MEMORY; }
  for (int64_t u = 0; u < n; ++u) out->truth[u] = uint32_t(u * k / n);
  return RAK_OK;
}

rak_status rak_gen_lattice(int64_t width, int64_t height, double p_delete, double shortcut_frac,
                           uint64_t seed, int threads, rak_host_csr *out) {
  if (!out || width < 1 || height < 1 || width * height >= (int64_t(1) << 31) || p_delete < 0 ||
      p_delete > 1 || shortcut_frac < 0)
    return RAK_ERR_INVALID_ARGUMENT;
  clear(out);
  Threads th(threads);
  const int64_t n = width * height;
  const int64_t eh = (width - 1) * height, grid = eh + width * (height - 1);
  const int64_t shortcuts = int64_t(std::llround(double(grid) * shortcut_frac));
  const uint32_t del24 = uint32_t(std::lround(p_delete * 16777216.0));
  auto gen = [=](int64_t i, uint32_t &u, uint32_t &v) {
    uint64_t h = rand64(seed, STREAM_LATTICE, uint64_t(i));
    if (i < grid) {
      if (uint32_t(h >> 40) < del24) return false;
      if (i < eh) { int64_t y = i / (width - 1), x = i % (width - 1); u = uint32_t(y * width + x); v = u + 1; }
      else { int64_t j = i - eh; u = uint32_t(j); v = uint32_t(j + width); }
      return true;
    }
    u = below(h, uint64_t(n));
    v = below(rand64(seed, STREAM_LATTICE + 16, uint64_t(i)), uint64_t(n));
    return true;
  };
  return build_symmetric(n, grid + shortcuts, gen, out);
}

void rak_host_csr_free(rak_host_csr *g) {
  if (!g) return;
  std::free(g->offsets);
  std::free(g->targets);
  std::free(g->weights);
  std::free(g->truth);
  clear(g);
}

}  // extern "C"
