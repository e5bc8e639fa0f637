// ref_bridge.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own CPU implementation (headers under the reference's inc/, included
// in place by oracle/Makefile; nothing is copied) into oracle/_ref/libref_cpu.so, exposing plain
// C entry points so the tests can pin the C restatement (rak_oracle.c) against the reference
// itself, and so bench.py can time the reference's CPU path on the host cores.
//
// The reference's algorithms take a graph type G; ShiftedCsr presents a caller's 0-based CSR to
// them with every vertex id shifted by one and vertex 0 absent, which is how the reference's MTX
// reader numbers vertices (inc/mtx.hxx:213,238). That matters because GVE-LPA treats label 0 as
// "no community" (inc/rak.hxx:216-220,252) and the sketch keys start at 0 (inc/rakLowmem.hxx:29).
#define BUILD 0
#define OPENMP 1
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <array>
#include <numeric>
#include <vector>
#include <omp.h>
#include "_main.hxx"
#include "Graph.hxx"
#include "mtx.hxx"
#include "symmetrize.hxx"
#include "properties.hxx"
#include "rak.hxx"
#include "rakLowmem.hxx"

using std::array;
using std::vector;

namespace {

struct ShiftedCsr {
  using key_type = uint32_t;
  using vertex_value_type = None;
  using edge_value_type = float;
  int64_t n;
  const int64_t *off;
  const uint32_t *tgt;
  const float *wt;

  size_t span() const noexcept { return size_t(n) + 1; }
  size_t order() const noexcept { return size_t(n); }
  size_t size() const noexcept { return size_t(off[n]); }
  bool hasVertex(uint32_t u) const noexcept { return u >= 1 && int64_t(u) <= n; }
  size_t degree(uint32_t u) const noexcept { return hasVertex(u) ? size_t(off[u] - off[u - 1]) : 0; }
  template <class F> void forEachVertexKey(F f) const noexcept {
    for (int64_t u = 1; u <= n; ++u) f(uint32_t(u));
  }
  template <class F> void forEachEdge(uint32_t u, F f) const noexcept {
    if (!hasVertex(u)) return;
    for (int64_t i = off[u - 1]; i < off[u]; ++i) f(uint32_t(tgt[i] + 1), wt ? wt[i] : 1.0f);
  }
  template <class F> void forEachEdgeKey(uint32_t u, F f) const noexcept {
    if (!hasVertex(u)) return;
    for (int64_t i = off[u - 1]; i < off[u]; ++i) f(uint32_t(tgt[i] + 1));
  }
};

// Shifted membership (index 1..n, values 1..n) -> 0-based labels.
void unshift(const vector<uint32_t> &m, int64_t n, uint32_t *labels) {
  for (int64_t u = 0; u < n; ++u) labels[u] = m[u + 1] - 1;
}

template <bool MULTI, bool RESCAN, size_t SLOTS>
int run_lowmem(const ShiftedCsr &x, double tol, int maxit, int repeat, uint32_t *labels, float *time_ms) {
  auto r = rakLowmemStaticOmp<MULTI, RESCAN, SLOTS>(x, RakOptions(repeat, tol, maxit));
  unshift(r.membership, x.n, labels);
  if (time_ms) *time_ms = r.time;
  return r.iterations;
}

// Synchronous driver over the reference's per-vertex functions: each decision reads the frozen
// snapshot, keys and weights start cleared for every vertex, and the move rule is the
// reference's (w>0 && c!=d, inc/rakLowmem.hxx:203). Marks go to the next frontier.
template <size_t SLOTS, bool RESCAN>
uint64_t sync_step_mg(const ShiftedCsr &x, bool pickless, const vector<uint32_t> &prev,
                      const uint8_t *aff_prev, uint32_t *next, uint8_t *aff_next) {
  uint64_t changed = 0;
  for (int64_t u = 1; u <= x.n; ++u) {
    if (!aff_prev[u - 1]) continue;
    array<uint32_t, SLOTS> mcs{};
    array<float, SLOTS> mws{};
    rakLowmemClearScanW(mws);
    rakLowmemScanCommunitiesW(mcs, mws, x, uint32_t(u), prev);
    auto cw = rakLowmemChooseCommunityW<false, RESCAN>(mws, x, uint32_t(u), mcs, prev);
    uint32_t c = cw.first, d = prev[u];
    float w = cw.second;
    if (!(w > 0 && c != d)) continue;
    if (pickless && c > d) continue;
    next[u - 1] = c - 1; ++changed;
    x.forEachEdgeKey(uint32_t(u), [&](uint32_t v) { if (v != uint32_t(u)) aff_next[v - 1] = 1; });
  }
  return changed;
}

uint64_t sync_step_bm(const ShiftedCsr &x, bool pickless, const vector<uint32_t> &prev,
                      const uint8_t *aff_prev, uint32_t *next, uint8_t *aff_next) {
  uint64_t changed = 0;
  for (int64_t u = 1; u <= x.n; ++u) {
    if (!aff_prev[u - 1]) continue;
    auto cw = rakLowmemScanCommunitiesMajority(x, uint32_t(u), prev);
    uint32_t c = cw.first, d = prev[u];
    float w = cw.second;
    if (!(w > 0 && c != d)) continue;
    if (pickless && c > d) continue;
    next[u - 1] = c - 1; ++changed;
    x.forEachEdgeKey(uint32_t(u), [&](uint32_t v) { if (v != uint32_t(u)) aff_next[v - 1] = 1; });
  }
  return changed;
}

}  // namespace

extern "C" {

// rakLowmemStaticOmp<MULTI,RESCAN,SLOTS> (inc/rakLowmem.hxx:277-284). slots==1 runs the
// Boyer-Moore variant (MULTI=false). Returns iterations, or -1 for an unsupported slot count.
int ref_lowmem_omp(int64_t n, const int64_t *off, const uint32_t *tgt, const float *wt, int slots,
                   int rescan, double tol, int maxit, int threads, int repeat, uint32_t *labels,
                   float *time_ms) {
  if (threads > 0) omp_set_num_threads(threads);
  ShiftedCsr x{n, off, tgt, wt};
  if (slots == 1) return run_lowmem<false, false, 8>(x, tol, maxit, repeat, labels, time_ms);
#define RL(S) \
  if (slots == S) return rescan ? run_lowmem<true, true, S>(x, tol, maxit, repeat, labels, time_ms) \
                                : run_lowmem<true, false, S>(x, tol, maxit, repeat, labels, time_ms);
  RL(2) RL(4) RL(8) RL(16) RL(32)
#undef RL
  return -1;
}

// rakStaticOmp (inc/rak.hxx:320-327), GVE-LPA with per-thread dense hashtables.
int ref_gve_omp(int64_t n, const int64_t *off, const uint32_t *tgt, const float *wt, double tol,
                int maxit, int threads, int repeat, uint32_t *labels, float *time_ms) {
  if (threads > 0) omp_set_num_threads(threads);
  ShiftedCsr x{n, off, tgt, wt};
  auto r = rakStaticOmp(x, RakOptions(repeat, tol, maxit));
  unshift(r.membership, n, labels);
  if (time_ms) *time_ms = r.time;
  return r.iterations;
}

// A bounded sample of the reference's first iteration, for timing on the host cores: its own setup
// function rakLowmemInvokeOmp<MULTI,RESCAN,SLOTS> (inc/rakLowmem.hxx:226-262) with the hooks of
// rakLowmemStaticOmp (:277-284: labels initialised by rakInitializeOmpW, every vertex marked
// affected) except that the "is vertex allowed to be updated" hook admits every stride-th vertex
// (0-based ids 0, stride, 2*stride, ...), and one iteration. Returns the traversed edges (the
// admitted vertices' degrees, summed outside the timed region); *time_ms is the reference's own
// measureDuration of the run. -1 for an unsupported slot count.
int64_t ref_lowmem_omp_sample(int64_t n, const int64_t *off, const uint32_t *tgt, const float *wt, int slots,
                              int rescan, int64_t stride, int threads, float *time_ms) {
  if (threads > 0) omp_set_num_threads(threads);
  if (stride < 1) stride = 1;
  ShiftedCsr x{n, off, tgt, wt};
  int64_t edges = 0;
  for (int64_t u = 0; u < n; u += stride) edges += off[u + 1] - off[u];
  const RakOptions o(1, 0.0, 1);
  using FLAG = char;
  auto fi = [&](auto &vcom) { rakInitializeOmpW(vcom, x); };
  auto fm = [](auto &vaff, auto &vcs, auto &vcout, const auto &vcom) { fillValueOmpU(vaff, FLAG(1)); };
  auto fa = [=](auto u) { return (int64_t(u) - 1) % stride == 0; };
  float t = -1;
  if (slots == 1) t = rakLowmemInvokeOmp<false, false, 8>(x, o, fi, fm, fa).time;
#define RS(S)                                                                 \
  else if (slots == S) t = rescan ? rakLowmemInvokeOmp<true, true, S>(x, o, fi, fm, fa).time \
                                  : rakLowmemInvokeOmp<true, false, S>(x, o, fi, fm, fa).time;
  RS(2) RS(4) RS(8) RS(16) RS(32)
#undef RS
  else return -1;
  if (time_ms) *time_ms = t;
  return edges;
}

// The same bounded sample of GVE-LPA's first iteration: rakInvokeOmp (inc/rak.hxx:272-310) with the
// hooks of rakStaticOmp (:320-327) except for the same every-stride-th-vertex "allowed" hook.
int64_t ref_gve_omp_sample(int64_t n, const int64_t *off, const uint32_t *tgt, const float *wt, int64_t stride,
                           int threads, float *time_ms) {
  if (threads > 0) omp_set_num_threads(threads);
  if (stride < 1) stride = 1;
  ShiftedCsr x{n, off, tgt, wt};
  int64_t edges = 0;
  for (int64_t u = 0; u < n; u += stride) edges += off[u + 1] - off[u];
  const RakOptions o(1, 0.0, 1);
  using FLAG = char;
  auto fi = [&](auto &vcom) { rakInitializeOmpW(vcom, x); };
  auto fm = [](auto &vaff, auto &vcs, auto &vcout, const auto &vcom) { fillValueOmpU(vaff, FLAG(1)); };
  auto fa = [=](auto u) { return (int64_t(u) - 1) % stride == 0; };
  const float t = rakInvokeOmp(x, o, fi, fm, fa).time;
  if (time_ms) *time_ms = t;
  return edges;
}

// modularityBy (inc/properties.hxx:177-192) with M = edgeWeightOmp(x)/2 as main.cxx:61 does.
double ref_modularity(int64_t n, const int64_t *off, const uint32_t *tgt, const float *wt,
                      const uint32_t *labels) {
  ShiftedCsr x{n, off, tgt, wt};
  double M = edgeWeightOmp(x) / 2;
  if (!(M > 0)) return 0.0;
  return modularityBy(x, [&](uint32_t u) { return labels[u - 1] + 1; }, M, 1.0);
}

// One synchronous iteration built from the reference's per-vertex functions.
// Returns changed count, or -1 for an unsupported slot count.
int64_t ref_sync_step(int64_t n, const int64_t *off, const uint32_t *tgt, const float *wt, int slots,
                      int rescan, int pickless, const uint32_t *vcom_prev, const uint8_t *aff_prev,
                      uint32_t *vcom_next, uint8_t *aff_next) {
  ShiftedCsr x{n, off, tgt, wt};
  vector<uint32_t> prev(size_t(n) + 1, 0);
  for (int64_t u = 0; u < n; ++u) { prev[u + 1] = vcom_prev[u] + 1; vcom_next[u] = vcom_prev[u]; aff_next[u] = 0; }
  bool pl = pickless != 0;
  if (slots == 1) return int64_t(sync_step_bm(x, pl, prev, aff_prev, vcom_next, aff_next));
#define SS(S) \
  if (slots == S) return int64_t(rescan ? sync_step_mg<S, true>(x, pl, prev, aff_prev, vcom_next, aff_next) \
                                        : sync_step_mg<S, false>(x, pl, prev, aff_prev, vcom_next, aff_next));
  SS(2) SS(4) SS(8) SS(16) SS(32)
#undef SS
  return -1;
}

// Feeds a stream of (community, weight) pairs through the reference's Misra-Gries accumulate
// (rakLowmemScanCommunityU, inc/rakLowmem.hxx:63-89) from cleared keys and weights, or through
// the Boyer-Moore rule of rakLowmemScanCommunitiesMajority (:115-128) when slots == 1, and
// returns the final slots (0-based keys; 0xFFFFFFFF for a key never set).
int ref_sketch_stream(int slots, int64_t len, const uint32_t *comm, const float *wts, uint32_t *keys_out,
                      float *w_out) {
  vector<uint32_t> vcom(size_t(len) + 1);
  for (int64_t i = 0; i < len; ++i) vcom[size_t(i)] = comm[i] + 1;
  const uint32_t u = 0xFFFFFFFFu;  // never equal to a stream index, so no edge counts as a self-loop
  if (slots == 1) {
    // A star: vertex 0 (shifted: 1) with one edge to each stream position i (shifted: i+2).
    vector<int64_t> off(size_t(len) + 2, len);
    off[0] = 0;
    vector<uint32_t> tgt(static_cast<size_t>(len), 0u);
    for (int64_t i = 0; i < len; ++i) tgt[size_t(i)] = uint32_t(i + 1);
    ShiftedCsr x{len + 1, off.data(), tgt.data(), wts};
    vector<uint32_t> vc(size_t(len) + 2, 0);
    for (int64_t i = 0; i < len; ++i) vc[size_t(i) + 2] = comm[i] + 1;
    auto cw = rakLowmemScanCommunitiesMajority(x, uint32_t(1), vc);
    keys_out[0] = cw.first - 1; w_out[0] = cw.second;
    return 0;
  }
#define ST(S) \
  if (slots == S) { \
    array<uint32_t, S> mcs{}; array<float, S> mws{}; \
    for (int64_t i = 0; i < len; ++i) rakLowmemScanCommunityU<false>(mcs, mws, u, uint32_t(i), wts[i], vcom); \
    for (int j = 0; j < S; ++j) { keys_out[j] = mcs[j] - 1; w_out[j] = mws[j]; } \
    return 0; \
  }
  ST(2) ST(4) ST(8) ST(16) ST(32)
#undef ST
  return -1;
}

// The reference driver's graph loading (main.cxx:116-119): readMtxOmpW into DiGraph<uint32_t, None,
// float>, then symmetrizeOmpU unless the caller says the file is symmetric. The result comes back
// 0-based (vertex k+1 of the reference is k here), targets sorted per vertex. Two passes: with
// off == nullptr only *n and *m are set.
int ref_read_mtx(const char *path, int weighted, int symmetrize, int64_t *n, int64_t *m, int64_t *off,
                 uint32_t *tgt, float *wt) {
  DiGraph<uint32_t, None, float> x;
  readMtxOmpW(x, path, weighted != 0);
  if (symmetrize) symmetrizeOmpU(x);
  const int64_t span = int64_t(x.span());
  *n = span > 0 ? span - 1 : 0;
  *m = int64_t(x.size());
  if (!off) return 0;
  int64_t e = 0;
  off[0] = 0;
  for (int64_t u = 1; u < span; ++u) {
    x.forEachEdge(uint32_t(u), [&](auto v, auto w) {
      tgt[e] = uint32_t(v) - 1;
      if (wt) wt[e] = float(w);
      ++e;
    });
    off[u] = e;
  }
  return 0;
}

// The vertex order of the reference's GPU entry (rakLowmemPartitionVerticesCudaU,
// inc/rakLowmemCuda.hxx:505-519, on vertexKeys(x)): keys in order, std::partition by degree < 4,
// then the remainder by degree < 128. That header needs the CUDA toolchain, so the two calls are
// restated here with the same predicates on the same standard library; 0-based ids (the
// reference's keys are these + 1, which does not change the order).
void ref_vertex_order(int64_t n, const int64_t *off, uint32_t *ks) {
  vector<uint32_t> k(static_cast<size_t>(n));
  std::iota(k.begin(), k.end(), 0u);
  auto fl = [&](uint32_t v) { return off[v + 1] - off[v] < 4; };
  auto fm = [&](uint32_t v) { return off[v + 1] - off[v] < 128; };
  auto il = std::partition(k.begin(), k.end(), fl);
  std::partition(il, k.end(), fm);
  std::copy(k.begin(), k.end(), ks);
}

}  // extern "C"
