// rak_lpa.cuh -- the persistent label-propagation kernel (all iterations in one cooperative
// launch) for νMG-LPA (S >= 2 Misra-Gries slots) and νBM-LPA (S == 1).
//
// Reference path replaced: rakLowmemLoopCuU (inc/rakLowmemCuda.hxx:469-490) and the move kernels
// it launches every iteration -- rakLowmemMgMoveIterationGroupCukU (:269-317),
// rakLowmemMgMoveIterationBlockCukU (:362-419), rakLowmemBmMoveIterationThreadCukU (:138-161),
// rakLowmemBmMoveIterationBlockCukU (:198-229) -- plus the per-iteration changed-count reset
// (fillValueCuW, :477) and blocking read-back (:486). Here the changed count, the traversed-edge
// count and the convergence test stay on the device; iterations are separated by a bounded grid
// barrier instead of kernel launches and host round trips.
//
// Work is a list of items over the plan's regions (rak_internal.hpp), heaviest first; warps take
// the next item from a per-iteration counter, so the load balances dynamically. Sketches live in
// registers, one per lane.
#pragma once
#include <map>
#include <mutex>
#include <utility>

#include "rak_device.cuh"
#include "rak_internal.hpp"

// Edges loaded ahead per lane in the scan pipeline, and the resident blocks per SM the register
// budget is sized for. Four blocks (64 registers; the asynchronous instantiations spill a few
// hundred bytes) against three (80 registers), measured on B200 on renumbered resident graphs, one
// box, runs alternated: R-MAT s27 100.5-100.7 vs 102.3-102.4 ms at lower clocks, s24 ef32 weighted
// 30.2 vs 31.4 ms, 2D lattice 2^25 9.0 vs 9.8 ms (on the graphs as given, earlier, four blocks were
// 1-5% slower): the loads in flight of the extra warps pay for the spills.
#ifndef RAK_SCAN_BATCH
#define RAK_SCAN_BATCH 4
#endif
#ifndef RAK_MIN_BLOCKS
#define RAK_MIN_BLOCKS 4
#endif

namespace rak {

struct Counters {
  unsigned long long edges;
  unsigned long long moved_edges;
  unsigned int changed;
  unsigned int processed;
};

// How an asynchronous iteration treats the frontier (LpaArgs::dense_moved_edges). all: every
// vertex is processed, whatever its flag (the previous iteration marked no neighbours); nomark:
// moved vertices mark no neighbours (the next iteration processes every vertex). Both false in
// the other modes and in batches: the reference's pruning, flags marked by every move.
struct Phase {
  bool all;
  bool nomark;
};

template <class O>
struct G_ {
  const O *off;
  const uint32_t *tgt;
  const float *wt;
};

// Edge-stream loads (targets, weights): non-coherent loads. RAK_STREAM_HINT=1 gives them an L2
// evict-first cache policy (an operand of the load instruction, not a setting of the GPU), meant to
// leave L2 capacity to the label gathers; measured on B200 it was 2-3% slower (R-MAT scale 27: 116
// vs 119 G edges/s; scale 24 weighted: 126 vs 128), so it is off.
#ifndef RAK_STREAM_HINT
#define RAK_STREAM_HINT 0
#endif
__device__ __forceinline__ uint64_t l2_stream_policy() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// RAK_L1_HINTS=1: edge-stream loads allocate in L1 as evict-first and label gathers as evict-last,
// so the streamed edge lines leave L1 before the labels that neighbours share.
#ifndef RAK_L1_HINTS
#define RAK_L1_HINTS 0
#endif
__device__ __forceinline__ uint32_t ld_edge(const uint32_t *p) {
#if RAK_L1_HINTS
  uint32_t v;
  asm("ld.global.nc.L1::evict_first.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
#elif RAK_STREAM_HINT
  uint32_t v;
  asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(l2_stream_policy()));
  return v;
#else
  return __ldg(p);
#endif
}
__device__ __forceinline__ float ld_weight(const float *p) {
#if RAK_L1_HINTS
  float v;
  asm("ld.global.nc.L1::evict_first.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
#elif RAK_STREAM_HINT
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(l2_stream_policy()));
  return v;
#else
  return __ldg(p);
#endif
}

// Label gathers (neighbour labels, which change during the launch: plain coherent loads).
// RAK_LABEL_HINT=1 gives them an L2 evict-last cache policy (an operand of the load instruction):
// when the label array is larger than L2, the lines of frequently read labels then outlast the
// streamed edge lines; RAK_LABEL_HINT=2 reads them from L2 only (not cached in L1).
#ifndef RAK_LABEL_HINT
#define RAK_LABEL_HINT 0
#endif
__device__ __forceinline__ uint64_t l2_keep_policy() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint32_t ld_label(const uint32_t *p) {
#if RAK_L1_HINTS && RAK_LABEL_HINT == 1
  uint32_t v;
  asm volatile("ld.global.L1::evict_last.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(l2_keep_policy()) : "memory");
  return v;
#elif RAK_L1_HINTS
  uint32_t v;
  asm volatile("ld.global.L1::evict_last.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
#elif RAK_LABEL_HINT == 1
  uint32_t v;
  asm volatile("ld.global.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(l2_keep_policy()) : "memory");
  return v;
#elif RAK_LABEL_HINT == 2
  return __ldcg(p);
#else
  return *p;
#endif
}

template <bool UNIT>
__device__ __forceinline__ float edge_w(const float *wt, int64_t e) {
  if constexpr (UNIT) return 1.0f;
  else return ld_weight(wt + e);
}

// Sequential sketch of edges e, e+st, ... < ee of u (self-loops skipped), in edge order.
// Software-pipelined in batches of four: the next batch's targets and weights are loaded while
// the current batch's labels are gathered and accumulated. Positions past the end are given the
// target u itself, which the self-loop rule skips. Labels are read with plain loads: they change
// during the launch.
template <int S, bool UNIT, int RULE>
__device__ __forceinline__ void scan_range(Sketch<S> &sk, uint32_t u, int64_t e, int64_t ee, int st,
                                           const uint32_t *tgt, const float *wt, const uint32_t *vin,
                                           uint32_t base) {
  constexpr int B = RAK_SCAN_BATCH;
  uint32_t t[B];
  float w[B];
#pragma unroll
  for (int j = 0; j < B; ++j) {
    const int64_t x = e + int64_t(j) * st;
    t[j] = x < ee ? base + ld_edge(tgt + x) : u;
    w[j] = x < ee ? edge_w<UNIT>(wt, x) : 0.0f;
  }
  while (e < ee) {
    uint32_t c[B];
#pragma unroll
    for (int j = 0; j < B; ++j) c[j] = ld_label(vin + t[j]);
    const int64_t en = e + int64_t(B) * st;
    uint32_t t2[B];
    float w2[B];
#pragma unroll
    for (int j = 0; j < B; ++j) {
      const int64_t x = en + int64_t(j) * st;
      t2[j] = x < ee ? base + ld_edge(tgt + x) : u;
      w2[j] = x < ee ? edge_w<UNIT>(wt, x) : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < B; ++j)
      if (t[j] != u) sk_acc<S, RULE>(sk, c[j], w[j]);
#pragma unroll
    for (int j = 0; j < B; ++j) { t[j] = t2[j]; w[j] = w2[j]; }
    e = en;
  }
}

// Neighbour marking reads a neighbour's flag before storing it when the launch asks for it
// (LpaArgs::mark_test, mark_test_for). The read goes through L1: most neighbours of a moved vertex
// are flagged already, and a flag line that L1 holds answers without a request to L2. In the
// synchronous modes the flags being set are only set during an iteration (and L1 is invalidated
// by the grid barrier's acquire), so a read can at worst miss a fresh mark and store it again. In
// the asynchronous mode a line L1 holds can also show a flag that another SM has cleared since
// (its vertex was processed); that neighbour is then not marked again for this move -- the same
// kind of lost update as the mode's unordered plain stores, measured with no change of modularity
// (R-MAT scale 24 and 27). RAK_MARK_FORCE=1/2 forces the test on/off (measurements).
#ifndef RAK_MARK_FORCE
#define RAK_MARK_FORCE 0
#endif
__device__ __forceinline__ uint32_t ld_flag_test(const uint8_t *p) { return *p; }

// ---- one lane per vertex: the edge list read in 16-byte vectors -------------------------------
//
// A lane that scans its own vertex of degree RAK_VEC_MIN_DEG or more reads 4 targets (and 4
// weights) per load instead of one: a warp issues a quarter of the edge-stream loads. Requires
// targets (and weights) at 16-byte aligned addresses (checked per launch, lane_vec_ok). Vector v covers edges 4v .. 4v+3; edges outside [e, ee) are masked with the
// target u itself, which the self-loop rule skips, so the lane accumulates exactly edges e .. ee-1
// in order, as scan_range with stride 1 does. Whole-vector loads stay inside [4*floor(e/4), ee);
// the last vector of a range whose end is not a multiple of 4 is read edge by edge.
template <bool UNIT>
__device__ __forceinline__ void load_vec4(int64_t v, int64_t ee, const uint32_t *tgt, const float *wt, uint4 &t4,
                                          float4 &w4) {
  const int64_t x0 = v << 2;
  if (x0 + 4 <= ee) {
#if RAK_L1_HINTS
    asm("ld.global.nc.L1::evict_first.v4.u32 {%0, %1, %2, %3}, [%4];"
        : "=r"(t4.x), "=r"(t4.y), "=r"(t4.z), "=r"(t4.w) : "l"(tgt + x0));
    if constexpr (!UNIT)
      asm("ld.global.nc.L1::evict_first.v4.f32 {%0, %1, %2, %3}, [%4];"
          : "=f"(w4.x), "=f"(w4.y), "=f"(w4.z), "=f"(w4.w) : "l"(wt + x0));
#else
    t4 = __ldg(reinterpret_cast<const uint4 *>(tgt) + v);
    if constexpr (!UNIT) w4 = __ldg(reinterpret_cast<const float4 *>(wt) + v);
#endif
  } else {
    t4.x = x0 < ee ? ld_edge(tgt + x0) : 0u;
    t4.y = x0 + 1 < ee ? ld_edge(tgt + x0 + 1) : 0u;
    t4.z = x0 + 2 < ee ? ld_edge(tgt + x0 + 2) : 0u;
    t4.w = 0u;   // x0 + 3 >= ee here
    if constexpr (!UNIT) {
      w4.x = x0 < ee ? ld_weight(wt + x0) : 0.0f;
      w4.y = x0 + 1 < ee ? ld_weight(wt + x0 + 1) : 0.0f;
      w4.z = x0 + 2 < ee ? ld_weight(wt + x0 + 2) : 0.0f;
      w4.w = 0.0f;
    }
  }
}

// Vector loads pay only on longer lists: a list's first and last vector carry masked positions,
// and the short lists of sparse graphs are mostly such vectors. Measured on B200 (vectors from
// degree 32 / always / never): 2D lattice 2^25 (degree ~4) 9.73 / 12.05 / 9.73 ms; R-MAT scale 25
// ef 4 8.22 / 8.51 / 8.10 ms; R-MAT scale 27 ef 16 128.0 / 128.5 / 130.2 ms; R-MAT scale 24 ef 32
// weighted 32.5 / 32.6 / 33.1 ms.
#ifndef RAK_VEC_MIN_DEG
#define RAK_VEC_MIN_DEG 32
#endif
__device__ __forceinline__ bool lane_vec_ok(const uint32_t *tgt, const float *wt) {
  return ((reinterpret_cast<uintptr_t>(tgt) | (wt ? reinterpret_cast<uintptr_t>(wt) : 0)) & 15u) == 0;
}

template <int S, bool UNIT, int RULE>
__device__ __forceinline__ void scan_lane(Sketch<S> &sk, uint32_t u, int64_t e, int64_t ee, const uint32_t *tgt,
                                          const float *wt, const uint32_t *vin, uint32_t base) {
  if (e >= ee) return;
  int64_t v = e >> 2;
  const int64_t vend = (ee + 3) >> 2;
  uint4 t4;
  float4 w4 = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
  load_vec4<UNIT>(v, ee, tgt, wt, t4, w4);
  for (; v < vend; ++v) {
    const int64_t x0 = v << 2;
    uint32_t t[4] = {t4.x, t4.y, t4.z, t4.w};
    float w[4] = {w4.x, w4.y, w4.z, w4.w};
    uint32_t c[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t x = x0 + j;
      t[j] = x >= e && x < ee ? base + t[j] : u;
      c[j] = t[j] != u ? ld_label(vin + t[j]) : NONE;
    }
    if (v + 1 < vend) load_vec4<UNIT>(v + 1, ee, tgt, wt, t4, w4);
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (t[j] != u) sk_acc<S, RULE>(sk, c[j], UNIT ? 1.0f : w[j]);
  }
}

// Neighbour marking of a moved vertex scanned by one lane (mark_range with stride 1), from 16-byte
// vectors of targets, two vectors in flight; TEST as in mark_range.
template <bool TEST>
__device__ __forceinline__ void mark_lane(uint32_t u, int64_t e, int64_t ee, const uint32_t *tgt, uint8_t *fout,
                                          uint32_t base) {
  if (e >= ee) return;
  const int64_t vend = (ee + 3) >> 2;
  float4 unused;
  for (int64_t v = e >> 2; v < vend; v += 2) {
    uint4 a4, b4 = make_uint4(0, 0, 0, 0);
    load_vec4<true>(v, ee, tgt, nullptr, a4, unused);
    if (v + 1 < vend) load_vec4<true>(v + 1, ee, tgt, nullptr, b4, unused);
    uint32_t t[8] = {a4.x, a4.y, a4.z, a4.w, b4.x, b4.y, b4.z, b4.w};
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int64_t x = (v << 2) + j;
      t[j] = x >= e && x < ee ? base + t[j] : u;
    }
    uint32_t f[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) f[j] = t[j] == u ? 1u : (TEST ? ld_flag_test(fout + t[j]) : 0u);
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (!f[j]) fout[t[j]] = 1;
  }
}

// Exact weights of the sketch keys in edge order (inc/rakLowmem.hxx:154-162), one lane.
template <int S, bool UNIT>
__device__ __forceinline__ void rescan_range(Sketch<S> &sk, uint32_t u, int64_t e, int64_t ee,
                                             const uint32_t *tgt, const float *wt, const uint32_t *vin,
                                             uint32_t base) {
#pragma unroll
  for (int i = 0; i < S; ++i) sk.w[i] = 0.0f;
  for (; e < ee; ++e) {
    const uint32_t v = base + ld_edge(tgt + e);
    if (v == u) continue;
    const uint32_t c = ld_label(vin + v);
    const float w = edge_w<UNIT>(wt, e);
#pragma unroll
    for (int i = 0; i < S; ++i)
      if (sk.k[i] == c) sk.w[i] = __fadd_rn(sk.w[i], w);
  }
}


// Marks neighbours e, e+st, ... < ee of a moved vertex u as affected (inc/rakCuda.hxx:95-103),
// except u itself (the reference CPU loop clears u after marking, inc/rakLowmem.hxx:203,209).
// Pipelined in batches of eight: the next batch's targets load while this batch is stored.
// test: store a flag only if it reads as clear (ld_flag_test). A random byte store costs the L2 a
// partial write, and most neighbours of a moved vertex are flagged already on large graphs; on
// small or sparse ones the read only lengthens the marking (mark_test_for chooses per launch).
template <bool TEST>
__device__ __forceinline__ void mark_range(uint32_t u, int64_t e, int64_t ee, int st, const uint32_t *tgt,
                                           uint8_t *fout, uint32_t base) {
  constexpr int MB = 8;
  uint32_t v[MB];
#pragma unroll
  for (int j = 0; j < MB; ++j) {
    const int64_t x = e + int64_t(j) * st;
    v[j] = x < ee ? base + ld_edge(tgt + x) : u;
  }
  while (e < ee) {
    uint32_t f[MB];
#pragma unroll
    for (int j = 0; j < MB; ++j) f[j] = v[j] == u ? 1u : (TEST ? ld_flag_test(fout + v[j]) : 0u);
    const int64_t en = e + int64_t(MB) * st;
    uint32_t v2[MB];
#pragma unroll
    for (int j = 0; j < MB; ++j) {
      const int64_t x = en + int64_t(j) * st;
      v2[j] = x < ee ? base + ld_edge(tgt + x) : u;
    }
#pragma unroll
    for (int j = 0; j < MB; ++j)
      if (!f[j]) fout[v[j]] = 1;
#pragma unroll
    for (int j = 0; j < MB; ++j) v[j] = v2[j];
    e = en;
  }
}


template <int S>
__device__ __forceinline__ bool mark_tested(const LpaArgs &a) {
  return RAK_MARK_FORCE == 1 || (RAK_MARK_FORCE == 0 && a.mark_test != 0);
}
template <int S>
__device__ __forceinline__ void mark_item(const LpaArgs &a, uint32_t u, int64_t e, int64_t ee, int st,
                                          const uint32_t *tgt, uint8_t *fout, uint32_t base) {
  if (mark_tested<S>(a)) mark_range<true>(u, e, ee, st, tgt, fout, base);
  else mark_range<false>(u, e, ee, st, tgt, fout, base);
}

// ---- edge tiles staged in shared memory by the bulk-copy engine (TMA) -------------------------
//
// Vertices scanned by a whole warp -- lane groups of 32 (region 1) and split-vertex chunks
// (region 0) -- read one contiguous edge range. With LpaArgs::stage the range is copied tile by
// tile into shared memory with 1-D bulk copies (cp.async.bulk, completion counted in bytes on an
// mbarrier), one tile ahead of the lanes, and the lanes read their edges there instead of loading
// them from global memory. Lane s still accumulates edges eb+s, eb+s+32, ... in that order, so the
// sketches are bit-identical to scan_range's. Bulk copies need 16-byte aligned addresses and sizes:
// the few edges before the range's first aligned address and after its last one are read from
// global memory directly, so no copy reads outside [eb, ee). The source is always this GPU's own
// memory; no copy uses a multicast form.
#ifndef RAK_STAGE
#define RAK_STAGE 1
#endif
constexpr int LPA_WARPS = 8;      // warps per block (256 threads)
constexpr int STG_TILE = 256;     // edges per tile (8 per lane): 16 KB of tiles per block (32 KB weighted)
constexpr int STG_STAGES = 2;     // tiles per warp: one in use, one in flight

// Dynamic shared memory of an lpa_run block that stages tiles: per warp STG_STAGES tiles of
// targets (and of weights, for weighted graphs), then one mbarrier per tile buffer.
__host__ __device__ constexpr size_t stage_bytes(bool unit) {
  return size_t(LPA_WARPS) * STG_STAGES * STG_TILE * 4 * (unit ? 1 : 2) + size_t(LPA_WARPS) * STG_STAGES * 8;
}

struct StageCtx {
  uint32_t *t;     // this warp's target buffers (STG_STAGES x STG_TILE)
  float *w;        // this warp's weight buffers (weighted graphs)
  uint32_t bar;    // shared-memory address of this warp's first mbarrier
  uint32_t phase;  // per buffer, the parity of the next completion to wait for (warp-uniform)
  bool on;         // staging in use for this launch
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_arrive(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// 1-D bulk copy global -> this CTA's shared memory, completing `bytes` on the mbarrier.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Waits for the completion of `parity` on an mbarrier, for at most timeout_ns of wall time. On
// expiry it records RAK_ERR_TIMEOUT and the launch's abort flag, as the grid barrier does (the
// launch then ends at its next barrier), and returns false: the caller reads that tile's edges
// from global memory instead.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, RunState *rs, long long timeout_ns) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try(bar, parity)) {
    if ((long long)(global_ns() - t0) > timeout_ns) {
      atomicCAS(&rs->error, 0u, 5u);
      atomicExch(&rs->abort, 1u);
      return false;
    }
  }
  return true;
}

// Lane 0 starts the copy of tile k of [cs, ce) into buffer k % STG_STAGES (all lanes call this).
template <bool UNIT>
__device__ __forceinline__ void stage_issue(const StageCtx &sc, int k, int64_t cs, int64_t ce, const uint32_t *tgt,
                                            const float *wt) {
  const int buf = k % STG_STAGES;
  const int64_t tb = cs + int64_t(k) * STG_TILE;
  const int64_t te = tb + STG_TILE < ce ? tb + STG_TILE : ce;
  const uint32_t bytes = te > tb ? uint32_t(te - tb) * 4u : 0u;
  const uint32_t bar = sc.bar + 8u * uint32_t(buf);
  fence_proxy_async_smem();  // this buffer's earlier reads come before the copy that refills it
  __syncwarp();
  if ((threadIdx.x & 31) == 0) {
    mbar_expect_arrive(bar, bytes * (UNIT ? 1u : 2u));
    if (bytes) {
      bulk_g2s(smem_u32(sc.t + buf * STG_TILE), tgt + tb, bytes, bar);
      if constexpr (!UNIT) bulk_g2s(smem_u32(sc.w + buf * STG_TILE), wt + tb, bytes, bar);
    }
  }
}

// Staged form of scan_range(sk, u, eb + lane, ee, 32, ...) for a range scanned by the whole warp.
// Every lane calls it with the same range (eb == ee: nothing to scan).
template <int S, bool UNIT, int RULE>
__device__ __forceinline__ void staged_scan(Sketch<S> &sk, StageCtx &sc, uint32_t u, int64_t eb, int64_t ee,
                                            const uint32_t *tgt, const float *wt, const uint32_t *vin, uint32_t base,
                                            RunState *rs, long long timeout_ns) {
  constexpr int B = RAK_SCAN_BATCH;
  const int lane = threadIdx.x & 31;
  // Copies cover [cs, ce): cs the first edge at a 16-byte aligned address at or after eb, ce the
  // last such boundary at or before ee. Tile k copies [cs + k*STG_TILE, min(cs + (k+1)*STG_TILE, ce));
  // the lanes take edges before cs in tile 0 and after ce in the last tile from global memory.
  int64_t cs = eb + int64_t(((16u - (uint32_t(reinterpret_cast<uintptr_t>(tgt + eb)) & 15u)) & 15u) >> 2);
  if (cs > ee) cs = ee;
  const int64_t ce = cs + ((ee - cs) & ~int64_t(3));
  int nt = ee > eb ? int((ee - cs + STG_TILE - 1) / STG_TILE) : 0;
  if (ee > eb && nt < 1) nt = 1;
  for (int k = 0; k < STG_STAGES && k < nt; ++k) stage_issue<UNIT>(sc, k, cs, ce, tgt, wt);
  int rel = int(eb - cs) + lane;   // the lane's next edge, relative to the current tile's first edge
  for (int k = 0; k < nt; ++k) {
    const int buf = k % STG_STAGES;
    const bool ok = mbar_wait(sc.bar + 8u * uint32_t(buf), (sc.phase >> buf) & 1u, rs, timeout_ns);
    sc.phase ^= 1u << buf;
    const int64_t tb = cs + int64_t(k) * STG_TILE;
    const uint32_t *bt = sc.t + buf * STG_TILE;
    const float *bw = sc.w + buf * STG_TILE;
    const bool whole = ok && k > 0 && tb + STG_TILE <= ce;   // every edge of the tile is in shared memory
    if (whole) {
#pragma unroll
      for (int b0 = 0; b0 < STG_TILE / 32; b0 += B) {
        uint32_t t[B], c[B];
        float w[B];
#pragma unroll
        for (int j = 0; j < B; ++j) {
          const int x = rel + (b0 + j) * 32;
          t[j] = base + bt[x];
          w[j] = UNIT ? 1.0f : bw[x];
        }
#pragma unroll
        for (int j = 0; j < B; ++j) c[j] = ld_label(vin + t[j]);
#pragma unroll
        for (int j = 0; j < B; ++j)
          if (t[j] != u) sk_acc<S, RULE>(sk, c[j], w[j]);
      }
      rel += STG_TILE;
    } else {
      // the first or last tile (or a tile whose copy gave up): edges outside the copy from global
      const int hi = k + 1 >= nt ? int(ee - tb) : STG_TILE;
      const int se = ok ? (tb + STG_TILE < ce ? STG_TILE : int(ce - tb)) : 0;
      // the lane consumes only its edges below hi, so that it enters the next tile at an offset
      // in [0, 32): the whole-tile path reads offsets up to that offset + STG_TILE - 32
      while (rel < hi) {
        const int left = (hi - rel + 31) >> 5;
        const int take = left < B ? left : B;
        uint32_t t[B], c[B];
        float w[B];
#pragma unroll
        for (int j = 0; j < B; ++j) {
          const int x = rel + j * 32;
          t[j] = u;
          w[j] = 0.0f;
          if (j < take) {
            const bool in = x >= 0 && x < se;
            t[j] = base + (in ? bt[x] : ld_edge(tgt + (tb + x)));
            if constexpr (UNIT) w[j] = 1.0f;
            else w[j] = in ? bw[x] : ld_weight(wt + (tb + x));
          }
        }
#pragma unroll
        for (int j = 0; j < B; ++j) c[j] = ld_label(vin + t[j]);
#pragma unroll
        for (int j = 0; j < B; ++j)
          if (t[j] != u) sk_acc<S, RULE>(sk, c[j], w[j]);
        rel += take * 32;
      }
    }
    rel -= STG_TILE;
    __syncwarp();
    if (k + STG_STAGES < nt) stage_issue<UNIT>(sc, k + STG_STAGES, cs, ce, tgt, wt);
  }
}

// Exact edge-order scan of u by the G lanes of one aligned group: lanes load G edges at a time,
// then every lane applies them in order from shuffles, so all lanes hold the same sketch as a
// single sequential scan would build (and, with rescan, the same exact weights).
template <int S, bool UNIT>
__device__ __forceinline__ void exact_group_scan(Sketch<S> &sk, uint32_t u, int64_t eb, int64_t ee, int G,
                                                 int g, int s, bool rescan, const uint32_t *tgt,
                                                 const float *wt, const uint32_t *vin, uint32_t base) {
  const unsigned gmask = G == 32 ? FULL : (((1u << G) - 1u) << (g * G));
  for (int pass = 0; pass < (rescan ? 2 : 1); ++pass) {
    if (pass == 1) {
#pragma unroll
      for (int i = 0; i < S; ++i) sk.w[i] = 0.0f;
    }
    for (int64_t e0 = eb; e0 < ee; e0 += G) {
      const int64_t e = e0 + s;
      uint32_t c = NONE;
      float w = 0.0f;
      int ok = 0;
      if (e < ee) {
        const uint32_t v = base + ld_edge(tgt + e);
        w = edge_w<UNIT>(wt, e);
        c = ld_label(vin + v);
        ok = v != u;
      }
      const int cnt = int(ee - e0 < G ? ee - e0 : G);
      for (int t = 0; t < cnt; ++t) {
        const uint32_t ct = __shfl_sync(gmask, c, g * G + t);
        const float wt_ = __shfl_sync(gmask, w, g * G + t);
        const int okt = __shfl_sync(gmask, ok, g * G + t);
        if (!okt) continue;
        if (pass == 0) {
          sk_acc(sk, ct, wt_);
        } else {
#pragma unroll
          for (int i = 0; i < S; ++i)
            if (sk.k[i] == ct) sk.w[i] = __fadd_rn(sk.w[i], wt_);
        }
      }
    }
  }
}

// Batches: a vertex's graph, whether that graph has converged, and its first vertex (the offset
// of the graph's local target ids). Single graphs: never finished, offset 0.
template <bool BATCH>
__device__ __forceinline__ bool graph_of(const LpaArgs &a, uint32_t u, uint32_t &gi, uint32_t &base) {
  if constexpr (BATCH) {
    gi = __ldg(a.gid + u);
    base = uint32_t(__ldg(a.vbase + gi));
    return a.gdone[gi] != 0;
  } else {
    gi = 0;
    base = 0;
    return false;
  }
}

template <bool BATCH>
__device__ __forceinline__ void count_move(const LpaArgs &a, uint32_t gi, int it) {
  if constexpr (BATCH) atomicAdd(a.gchanged + int64_t(it & 1) * a.ngraphs + gi, 1ull);
}

// CPU rule: w > 0 && c != d (inc/rakLowmem.hxx:203). GPU rule: the best weight is non-zero for
// Misra-Gries (inc/rakLowmemCuda.hxx:306), any candidate for Boyer-Moore (:152). Both: on pickless
// iterations no move to a larger label (:309, :153).
template <int S, int RULE>
__device__ __forceinline__ bool move_rule(float w, uint32_t c, uint32_t d, bool pickless) {
  const bool weight_ok = RULE == RULE_GPU ? (S == 1 || w != 0.0f) : w > 0.0f;
  return weight_ok && c != d && !(pickless && c > d);
}

// Argmax of a vertex's sketch under the launch's tie rule: hashed ties on iterations
// l < a.tie_until (Misra-Gries, CPU rules), else the rule set's own. u_local: the vertex's id within
// its graph, so a graph breaks its ties the same way alone and in a batch.
template <int S, int RULE>
__device__ __forceinline__ void choose(const LpaArgs &a, const Sketch<S> &sk, uint32_t u_local, int it, uint32_t &c,
                                       float &w) {
  if constexpr (S > 1 && RULE == RULE_CPU) {
    const int l = a.start_iter + it;
    if (l < a.tie_until) {
      sk_choose_hashed<S>(sk, u_local, uint32_t(l), c, w);
      return;
    }
  }
  sk_choose<S, RULE>(sk, c, w);
}

// Region 6: one lane per vertex. Items are collected into a per-warp queue of active vertices
// (inactive ones are settled at once), and the queue is processed 32 vertices at a time so every
// lane has work; region 6 is sorted by degree, so a batch holds vertices of similar degree.
template <int S, int MODE, class O, bool UNIT, bool BATCH>
__device__ __forceinline__ int lane_collect(const LpaArgs &a, const Regions &rg, int64_t local, const uint32_t *vin,
                                            uint32_t *vout, const uint8_t *fin, uint32_t *q, int qn, Phase ph) {
  const int lane = threadIdx.x & 31;
  const int64_t idx = local * 32 + lane;
  bool act = false;
  uint32_t u = 0;
  if (idx < rg.vcount[REG_LANE]) {
    u = __ldg(a.order + rg.vbegin[REG_LANE] + idx);
    uint32_t gi, base;
    act = (ph.all || fin[u] != 0) && !graph_of<BATCH>(a, u, gi, base);
    if constexpr (MODE != MODE_ASYNC)
      if (!act) vout[u] = vin[u];
  }
  const unsigned m = __ballot_sync(FULL, act);
  if (act) q[qn + __popc(m & ((1u << lane) - 1u))] = u;
  __syncwarp();
  return qn + __popc(m);
}

template <int S, int MODE, class O, bool UNIT, bool BATCH, int RULE>
__device__ __forceinline__ void lane_batch(const LpaArgs &a, const G_<O> &g, const uint32_t *q, int count,
                                           int it, bool pickless, const uint32_t *vin, uint32_t *vout,
                                           uint8_t *fin, uint8_t *fout, Counters &cnt, Phase ph) {
  const int lane = threadIdx.x & 31;
  if (lane >= count) return;
  const uint32_t u = q[lane];
  const uint32_t d = vin[u];
  uint32_t gi, base;
  graph_of<BATCH>(a, u, gi, base);
  const int64_t eb = int64_t(__ldg(g.off + u)), ee = int64_t(__ldg(g.off + u + 1));
  Sketch<S> sk;
  sk_clear<S, RULE>(sk, d);
  const bool vec = lane_vec_ok(g.tgt, g.wt) && ee - eb >= RAK_VEC_MIN_DEG;
  if (vec) scan_lane<S, UNIT, RULE>(sk, u, eb, ee, g.tgt, g.wt, vin, base);
  else scan_range<S, UNIT, RULE>(sk, u, eb, ee, 1, g.tgt, g.wt, vin, base);
  if constexpr (MODE == MODE_SYNC && S > 1)
    if (a.rescan) rescan_range<S, UNIT>(sk, u, eb, ee, g.tgt, g.wt, vin, base);
  uint32_t c;
  float w;
  choose<S, RULE>(a, sk, u - base, it, c, w);
  const bool moved = move_rule<S, RULE>(w, c, d, pickless);
  cnt.processed += 1;
  cnt.edges += (unsigned long long)(ee - eb);
  if constexpr (MODE == MODE_ASYNC) {
    fin[u] = 0;
    if (moved) vout[u] = c;
  } else {
    vout[u] = moved ? c : d;
  }
  if (moved) {
    cnt.changed += 1;
    cnt.moved_edges += (unsigned long long)(ee - eb);
    count_move<BATCH>(a, gi, it);
    if (ph.nomark) return;
    if (!vec) mark_item<S>(a, u, eb, ee, 1, g.tgt, fout, base);
    else if (mark_tested<S>(a)) mark_lane<true>(u, eb, ee, g.tgt, fout, base);
    else mark_lane<false>(u, eb, ee, g.tgt, fout, base);
  }
}

// Regions 1..5: aligned groups of G lanes per vertex.
template <int S, int MODE, class O, bool UNIT, bool BATCH, int RULE>
__device__ __forceinline__ void group_item(const LpaArgs &a, const Regions &rg, const G_<O> &g, int r, int64_t local,
                                           int it, bool pickless, const uint32_t *vin, uint32_t *vout,
                                           uint8_t *fin, uint8_t *fout, Counters &cnt, StageCtx &sc, Phase ph) {
  const int G = region_group(r);
  const int lane = threadIdx.x & 31, grp = lane / G, s = lane & (G - 1);
  const int64_t idx = local * (32 / G) + grp;
  const bool valid = idx < rg.vcount[r];
  uint32_t u = 0, d = 0, gi = 0, base = 0;
  int64_t eb = 0, ee = 0;
  bool active = false;
  if (valid) {
    u = __ldg(a.order + rg.vbegin[r] + idx);
    d = vin[u];
    active = (ph.all || fin[u] != 0) && !graph_of<BATCH>(a, u, gi, base);
    if (active) { eb = int64_t(__ldg(g.off + u)); ee = int64_t(__ldg(g.off + u + 1)); }
  }
  Sketch<S> sk;
  sk_clear<S, RULE>(sk, d);
  if constexpr (MODE == MODE_SYNC) {
    if (active) exact_group_scan<S, UNIT>(sk, u, eb, ee, G, grp, s, S > 1 && a.rescan, g.tgt, g.wt, vin, base);
  } else {
    if (sc.on && G == 32)   // one vertex per warp: the warp's range is uniform
      staged_scan<S, UNIT, RULE>(sk, sc, u, active ? eb : 0, active ? ee : 0, g.tgt, g.wt, vin, base,
                                 static_cast<RunState *>(a.rs), a.timeout_ns);
    else if (active)
      scan_range<S, UNIT, RULE>(sk, u, eb + s, ee, G, g.tgt, g.wt, vin, base);
    sk_tree<S, RULE>(sk, G);
  }
  uint32_t c;
  float w;
  choose<S, RULE>(a, sk, u - base, it, c, w);
  bool moved = active && move_rule<S, RULE>(w, c, d, pickless);
  moved = __shfl_sync(FULL, moved, grp * G);
  if (s == 0 && valid) {
    if (active) { cnt.processed += 1; cnt.edges += (unsigned long long)(ee - eb); }
    if constexpr (MODE == MODE_ASYNC) {
      if (active) fin[u] = 0;
      if (moved) vout[u] = c;
    } else {
      vout[u] = moved ? c : d;
    }
    if (moved) { cnt.changed += 1; cnt.moved_edges += (unsigned long long)(ee - eb); count_move<BATCH>(a, gi, it); }
  }
  if (moved && !ph.nomark) mark_item<S>(a, u, eb + s, ee, G, g.tgt, fout, base);
}

// Region 0: one chunk of a split vertex per item. In the synchronous exact mode chunk 0's warp
// scans the whole vertex in edge order and the other chunks do nothing. Otherwise each chunk's
// warp builds a partial sketch (lane-strided, tree-merged), stores it, and the last chunk to
// arrive merges all partial sketches in a fixed order and makes the move; its neighbours are
// marked in a second phase after the iteration's barrier.
template <int S, int MODE, class O, bool UNIT, bool BATCH, int RULE>
__device__ __forceinline__ void hub_item(const LpaArgs &a, const Regions &rg, const G_<O> &g, int64_t local, int it, bool pickless,
                                         const uint32_t *vin, uint32_t *vout, uint8_t *fin, uint8_t *fout,
                                         Counters &cnt, StageCtx &sc, Phase ph) {
  const int lane = threadIdx.x & 31;
  const uint32_t h = __ldg(a.chunk_hub + local);
  const int64_t first = __ldg(a.hub_first + h), nch = __ldg(a.hub_first + h + 1) - first, j = local - first;
  const uint32_t u = __ldg(a.order + rg.vbegin[REG_HUB] + h);
  const int64_t eb = int64_t(__ldg(g.off + u)), ee = int64_t(__ldg(g.off + u + 1));
  uint32_t gi, base;
  const bool gfin = graph_of<BATCH>(a, u, gi, base);  // stable within an iteration
  if constexpr (MODE == MODE_SYNC) {
    if (j != 0) return;
    const uint32_t d = vin[u];
    const bool active = fin[u] != 0 && !gfin;
    Sketch<S> sk;
    sk_clear<S, RULE>(sk, d);
    if (active) exact_group_scan<S, UNIT>(sk, u, eb, ee, 32, 0, lane, S > 1 && a.rescan, g.tgt, g.wt, vin, base);
    uint32_t c;
    float w;
    choose<S, RULE>(a, sk, u - base, it, c, w);
    const bool moved = active && move_rule<S, RULE>(w, c, d, pickless);
    if (lane == 0) {
      vout[u] = moved ? c : d;
      if (active) { cnt.processed += 1; cnt.edges += (unsigned long long)(ee - eb); }
      if (moved) { cnt.changed += 1; cnt.moved_edges += (unsigned long long)(ee - eb); count_move<BATCH>(a, gi, it); }
    }
    if (moved) mark_item<S>(a, u, eb + lane, ee, 32, g.tgt, fout, base);
    return;
  } else {
    bool active;
    if (gfin) {
      active = false;
    } else if constexpr (MODE == MODE_SPLIT) {
      active = fin[u] != 0;
    } else {
      // All chunks of u agree on whether u is processed this iteration: the first chunk to get
      // here decides from u's flag (and clears it); the others read the decision.
      unsigned int dec = 0;
      if (lane == 0) {
        const unsigned int tag = unsigned(it + 1);
        unsigned int cur = *(volatile unsigned int *)(a.hub_claim + h);
        if ((cur >> 1) != tag) {
          const unsigned int want = (tag << 1) | (ph.all || *(volatile uint8_t *)(fin + u) ? 1u : 0u);
          const unsigned int prev = atomicCAS(a.hub_claim + h, cur, want);
          if (prev == cur) {
            cur = want;
            if (want & 1u) fin[u] = 0;
          } else {
            cur = prev;
          }
        }
        dec = cur & 1u;
      }
      active = __shfl_sync(FULL, dec, 0) != 0;
    }
    // Boyer-Moore under the GPU rules starts every partial vote from u's label
    const uint32_t d0 = (S == 1 && RULE == RULE_GPU) ? vin[u] : NONE;
    Sketch<S> sk;
    sk_clear<S, RULE>(sk, d0);
    const int64_t cb = eb + j * a.hub_chunk, ce = cb + a.hub_chunk < ee ? cb + a.hub_chunk : ee;
    if (sc.on)   // active is the same on every lane
      staged_scan<S, UNIT, RULE>(sk, sc, u, active ? cb : 0, active ? ce : 0, g.tgt, g.wt, vin, base,
                                 static_cast<RunState *>(a.rs), a.timeout_ns);
    else if (active)
      scan_range<S, UNIT, RULE>(sk, u, cb + lane, ce, 32, g.tgt, g.wt, vin, base);
    sk_tree<S, RULE>(sk, 32);
    unsigned int last = 0;
    if (lane == 0) {
      if (active) {
        cnt.edges += (unsigned long long)(ce - cb);
#pragma unroll
        for (int i = 0; i < S; ++i) {
          a.sk_keys[local * S + i] = sk.k[i];
          a.sk_wts[local * S + i] = sk.w[i];
        }
      }
      __threadfence();
      last = atomicAdd(a.hub_arrive + h, 1u) == unsigned(nch - 1);
    }
    last = __shfl_sync(FULL, last, 0);
    if (!last) return;
    __threadfence();
    if (lane == 0) a.hub_arrive[h] = 0;
    const uint32_t d = vin[u];
    if (!active) {
      if (MODE != MODE_ASYNC && lane == 0) vout[u] = d;
      return;
    }
    Sketch<S> acc;
    sk_clear<S, RULE>(acc, d0);
    for (int64_t jj = lane; jj < nch; jj += 32) {
      uint32_t bk[S];
      float bw[S];
#pragma unroll
      for (int i = 0; i < S; ++i) {
        bk[i] = __ldcg(a.sk_keys + (first + jj) * S + i);
        bw[i] = __ldcg(a.sk_wts + (first + jj) * S + i);
      }
      sk_merge<S, RULE>(acc, bk, bw);
    }
    sk_tree<S, RULE>(acc, 32);
    if (lane == 0) {
      uint32_t c;
      float w;
      choose<S, RULE>(a, acc, u - base, it, c, w);
      const bool moved = move_rule<S, RULE>(w, c, d, pickless);
      cnt.processed += 1;
      if constexpr (MODE == MODE_ASYNC) {
        if (moved) vout[u] = c;
      } else {
        vout[u] = moved ? c : d;
      }
      if (moved) {
        cnt.changed += 1;
        cnt.moved_edges += (unsigned long long)(ee - eb);
        count_move<BATCH>(a, gi, it);
        a.hub_moved[h] = it;
        atomicAdd(a.stats + STATS_STRIDE * it + STAT_HUBS_MOVED, 1ull);
      }
    }
  }
}

// The rule set of a work item: the exact synchronous mode follows the CPU rules; the split-layout
// modes (asynchronous and synchronous split) either, per launch (a.gpu_rule).
#define RAK_BY_RULE(F, ARGS)                                                            \
  do {                                                                                 \
    if constexpr (MODE != MODE_SYNC) {                                                 \
      if (a.gpu_rule) F<S, MODE, O, UNIT, BATCH, RULE_GPU> ARGS;                       \
      else F<S, MODE, O, UNIT, BATCH, RULE_CPU> ARGS;                                  \
    } else {                                                                           \
      F<S, MODE, O, UNIT, BATCH, RULE_CPU> ARGS;                                       \
    }                                                                                  \
  } while (0)

template <int S, int MODE, class O, bool UNIT, bool BATCH>
__global__ void __launch_bounds__(256, RAK_MIN_BLOCKS) lpa_run(const LpaArgs a) {
  const G_<O> g{static_cast<const O *>(a.off), a.tgt, a.wt};
  RunState *rs = static_cast<RunState *>(a.rs);
  const int lane = threadIdx.x & 31;
  const int64_t gw = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  __shared__ unsigned long long blk[4];
  __shared__ Regions rg;  // copied once: indexed by region at run time
  __shared__ uint32_t lq[8][64];  // per-warp queue of active one-lane vertices
  if (threadIdx.x == 0) rg = a.rg;
  // staged edge tiles (not in the exact synchronous mode, which shuffles edges in order instead)
  StageCtx sc{};
  if constexpr (MODE != MODE_SYNC && RAK_STAGE) {
    extern __shared__ __align__(128) unsigned char lpa_dsm[];
    const int w = threadIdx.x >> 5;
    constexpr size_t tbytes = size_t(LPA_WARPS) * STG_STAGES * STG_TILE * 4;
    sc.t = reinterpret_cast<uint32_t *>(lpa_dsm) + size_t(w) * STG_STAGES * STG_TILE;
    sc.w = UNIT ? nullptr : reinterpret_cast<float *>(lpa_dsm + tbytes) + size_t(w) * STG_STAGES * STG_TILE;
    sc.bar = smem_u32(lpa_dsm + tbytes * (UNIT ? 1 : 2)) + 8u * uint32_t(w * STG_STAGES);
    sc.phase = 0;
    // the tiles and their mbarriers exist only in launches given the dynamic shared memory for them
    // (lpa_dynamic_smem); the launch's actual size is checked before any of it is touched
    uint32_t dyn_bytes;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn_bytes));
    const bool have = a.stage && dyn_bytes >= stage_bytes(UNIT);
    // targets and weights must share their 16-byte alignment (one copy range serves both)
    sc.on = have && (UNIT || ((reinterpret_cast<uintptr_t>(a.tgt) ^ reinterpret_cast<uintptr_t>(a.wt)) & 15u) == 0);
    if (have) {
      if (lane < STG_STAGES) mbar_init(sc.bar + 8u * uint32_t(lane), 1);
      fence_mbar_init();
      __syncwarp();
    }
  }
  unsigned int epoch = 0;
  // Dense iterations (asynchronous single-graph runs with LpaArgs::dense_moved_edges > 0): when
  // the vertices that moved in the previous iteration hold at least that many edges, this
  // iteration's moves mark no neighbours and the next iteration processes every vertex. Such a
  // frontier would hold nearly every vertex anyway, and the marking it saves is a re-read of each
  // moved vertex's edges plus a random flag access per edge. Decided from the previous iteration's
  // counter, which every block reads after the barrier, so all blocks agree.
  Phase ph{false, false};
  for (int it = 0; it < a.iters; ++it) {
    if (threadIdx.x < 4) blk[threadIdx.x] = 0;
    if constexpr (MODE == MODE_ASYNC && !BATCH) {
      ph.all = ph.nomark;
      ph.nomark = a.dense_moved_edges > 0 && it > 0 &&
                  __ldcg(a.stats + STATS_STRIDE * (it - 1) + STAT_MOVED_EDGES) >= a.dense_moved_edges;
      if (blockIdx.x == 0 && threadIdx.x == 0)
        a.stats[STATS_STRIDE * it + STAT_PHASE] = (ph.all ? 2ull : 0ull) | (ph.nomark ? 1ull : 0ull);
    }
    __syncthreads();
    const int l = a.start_iter + it;
    const bool pickless = a.pickless_step > 0 && l % a.pickless_step == 0;
    const bool odd = MODE != MODE_ASYNC && (it & 1);
    const uint32_t *vin = odd ? a.vcom1 : a.vcom0;
    uint32_t *vout = MODE == MODE_ASYNC ? a.vcom0 : (odd ? a.vcom0 : a.vcom1);
    uint8_t *fin = odd ? a.aff1 : a.aff0;
    uint8_t *fout = MODE == MODE_ASYNC ? a.aff0 : (odd ? a.aff0 : a.aff1);
    Counters cnt{0, 0, 0, 0};
    const int64_t total = rg.ibegin[NREG];
    unsigned long long *work = a.stats + STATS_STRIDE * it + STAT_WORK;
    uint32_t *q = lq[threadIdx.x >> 5];
    int qn = 0;
    for (;;) {
      unsigned long long got = 0;
      if (lane == 0) got = atomicAdd(work, 1ull);
      const int64_t item = int64_t(__shfl_sync(FULL, got, 0));
      if (item >= total) break;
      int r = 0;
      while (item >= rg.ibegin[r + 1]) ++r;
      const int64_t local = item - rg.ibegin[r];
      if (r == REG_LANE) {
        for (int64_t sb = 0; sb < rg.lane_item; ++sb) {
          const int64_t sub = local * rg.lane_item + sb;
          if (sub * 32 >= rg.vcount[REG_LANE]) break;
          qn = lane_collect<S, MODE, O, UNIT, BATCH>(a, rg, sub, vin, vout, fin, q, qn, ph);
          if (qn >= 32) {
            RAK_BY_RULE(lane_batch, (a, g, q, 32, it, pickless, vin, vout, fin, fout, cnt, ph));
            __syncwarp();
            if (lane < qn - 32) q[lane] = q[32 + lane];
            __syncwarp();
            qn -= 32;
          }
        }
      } else if (r == REG_HUB) {
        RAK_BY_RULE(hub_item, (a, rg, g, local, it, pickless, vin, vout, fin, fout, cnt, sc, ph));
      } else {
        RAK_BY_RULE(group_item, (a, rg, g, r, local, it, pickless, vin, vout, fin, fout, cnt, sc, ph));
      }
    }
    if (qn > 0) RAK_BY_RULE(lane_batch, (a, g, q, qn, it, pickless, vin, vout, fin, fout, cnt, ph));
    __syncwarp();
    const unsigned long long ch = warp_sum((unsigned long long)cnt.changed);
    const unsigned long long ed = warp_sum(cnt.edges);
    const unsigned long long pr = warp_sum((unsigned long long)cnt.processed);
    const unsigned long long me = warp_sum(cnt.moved_edges);
    if (lane == 0) {
      if (ch) atomicAdd(&blk[0], ch);
      if (ed) atomicAdd(&blk[1], ed);
      if (pr) atomicAdd(&blk[2], pr);
      if (me) atomicAdd(&blk[3], me);
    }
    __syncthreads();
    if (threadIdx.x < 4 && blk[threadIdx.x]) {
      const int slot = threadIdx.x == 3 ? STAT_MOVED_EDGES : int(threadIdx.x);
      atomicAdd(a.stats + STATS_STRIDE * it + slot, blk[threadIdx.x]);
    }
    if (!grid_barrier(rs, ++epoch, a.timeout_ns)) return;
    const unsigned long long changed = __ldcg(a.stats + STATS_STRIDE * it + STAT_CHANGED);
    const bool test = !pickless || a.check_on_pickless;
    // Batches finish when no graph is still running (decided in the per-graph phase below).
    const bool done = !BATCH && (it + 1 >= a.iters || (test && double(changed) / double(a.n) <= a.tolerance));
    // The synchronous split mode completes the next flags even on the last iteration, so a
    // single step returns them whole.
    if (MODE != MODE_SYNC && !ph.nomark && (!done || MODE == MODE_SPLIT) && a.nchunks > 0 &&
        __ldcg(a.stats + STATS_STRIDE * it + STAT_HUBS_MOVED) > 0) {
      // Second phase: neighbours of split vertices that moved this iteration.
      for (int64_t i = gw; i < a.nchunks; i += nw) {
        const uint32_t h = __ldg(a.chunk_hub + i);
        if (__ldcg(a.hub_moved + h) != it) continue;
        const uint32_t u = __ldg(a.order + rg.vbegin[REG_HUB] + h);
        const int64_t eb = int64_t(__ldg(g.off + u)), ee = int64_t(__ldg(g.off + u + 1));
        const int64_t j = i - __ldg(a.hub_first + h);
        const int64_t cb = eb + j * a.hub_chunk, ce = cb + a.hub_chunk < ee ? cb + a.hub_chunk : ee;
        uint32_t gi, base;
        graph_of<BATCH>(a, u, gi, base);
        mark_range<true>(u, cb + lane, ce, 32, g.tgt, fout, base);
      }
    }
    if constexpr (BATCH) {
      // Per-graph convergence, each graph by one thread: the rule of the single-graph loop applied
      // to the graph's own changed count and vertex count; also clears the graph's counter for the
      // iteration after next.
      const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
      unsigned int run = 0;
      for (int64_t gi = tid; gi < a.ngraphs; gi += nt) {
        if (a.gdone[gi]) continue;
        const int64_t ng = a.vbase[gi + 1] - a.vbase[gi];
        const unsigned long long c = __ldcg(a.gchanged + int64_t(it & 1) * a.ngraphs + gi);
        if (ng == 0 || it + 1 >= a.iters || (test && double(c) / double(ng) <= a.tolerance)) {
          a.gdone[gi] = 1;
          a.giters[gi] = it + 1;
        } else {
          ++run;
        }
        a.gchanged[int64_t((it + 1) & 1) * a.ngraphs + gi] = 0ull;
      }
      run = warp_sum(run);
      if (lane == 0 && run) atomicAdd(a.running + it, run);
      if constexpr (MODE != MODE_ASYNC) {
        uint4 *f4 = reinterpret_cast<uint4 *>(fin);
        const int64_t n16 = a.n >> 4;
        for (int64_t i = tid; i < n16; i += nt) f4[i] = make_uint4(0, 0, 0, 0);
        for (int64_t i = (n16 << 4) + tid; i < a.n; i += nt) fin[i] = 0;
      }
      if (!grid_barrier(rs, ++epoch, a.timeout_ns)) return;
      if (__ldcg(a.running + it) == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) rs->iterations = unsigned(it + 1);
        return;
      }
      continue;
    }
    if (done) {
      if (blockIdx.x == 0 && threadIdx.x == 0) rs->iterations = unsigned(it + 1);
      return;
    }
    if constexpr (MODE != MODE_ASYNC) {
      // The flags just read become next iteration's output: clear them.
      const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
      uint4 *f4 = reinterpret_cast<uint4 *>(fin);
      const int64_t n16 = a.n >> 4;
      for (int64_t i = tid; i < n16; i += nt) f4[i] = make_uint4(0, 0, 0, 0);
      for (int64_t i = (n16 << 4) + tid; i < a.n; i += nt) fin[i] = 0;
      if (!grid_barrier(rs, ++epoch, a.timeout_ns)) return;
    }
  }
}

// Dynamic shared memory of an lpa_run launch: the staged edge tiles, when the launch stages edges.
// Without staging the launch takes none, which leaves the SM's L1 cache its full size for the
// label gathers (shared memory and L1 share the SM's 256 KB).
inline size_t lpa_dynamic_smem(int mode, bool unit, bool stage) {
  return (mode != MODE_SYNC && RAK_STAGE && stage) ? stage_bytes(unit) : 0;
}

// The kernel instantiation for a launch and its resident blocks per SM, cached per (function,
// device). The first query of an instantiation loads its module (CUDA loads modules lazily, which
// can take a millisecond), so runs resolve before their timed region (prepare_lpa).
template <int S>
cudaError_t resolve_lpa_slots(int mode, bool off64, bool unit, bool batch, bool stage, const void **fn_out,
                              int *per_sm_out) {
  const void *fn = nullptr;
#define RAK_PICK(M, O, U, B)                                                          \
  if (mode == M && off64 == (sizeof(O) == 8) && unit == U && batch == B)             \
    fn = reinterpret_cast<const void *>(&lpa_run<S, M, O, U, B>);
#define RAK_PICK_MODE(M)                                                             \
  RAK_PICK(M, int32_t, false, false) RAK_PICK(M, int32_t, true, false)                \
  RAK_PICK(M, int64_t, false, false) RAK_PICK(M, int64_t, true, false)                \
  RAK_PICK(M, int64_t, false, true) RAK_PICK(M, int64_t, true, true)
  RAK_PICK_MODE(MODE_ASYNC) RAK_PICK_MODE(MODE_SYNC) RAK_PICK_MODE(MODE_SPLIT)
#undef RAK_PICK_MODE
#undef RAK_PICK
  if (!fn) return cudaErrorInvalidValue;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> cache;   // (kernel, device * 2 + stage)
  {
    std::lock_guard<std::mutex> lk(mu);
    const auto it = cache.find({fn, dev * 2 + (stage ? 1 : 0)});
    if (it != cache.end()) {
      *fn_out = fn;
      *per_sm_out = it->second;
      return cudaSuccess;
    }
  }
  int per_sm = 0;
  const size_t dyn = lpa_dynamic_smem(mode, unit, stage);
  if (dyn > 0 && (e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn))) != cudaSuccess)
    return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, dyn)) != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  std::lock_guard<std::mutex> lk(mu);
  cache[{fn, dev * 2 + (stage ? 1 : 0)}] = per_sm;
  *fn_out = fn;
  *per_sm_out = per_sm;
  return cudaSuccess;
}

template <int S>
cudaError_t launch_lpa_slots(const LpaArgs &a, int mode, bool off64, bool batch, cudaStream_t st, int *grid_out) {
  const void *fn = nullptr;
  int per_sm = 0, dev = 0, sms = 0;
  cudaError_t e = resolve_lpa_slots<S>(mode, off64, a.wt == nullptr, batch, a.stage != 0, &fn, &per_sm);
  if (e != cudaSuccess) return e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  const int64_t warps_needed = a.rg.ibegin[NREG] > 0 ? a.rg.ibegin[NREG] : 1;
  int64_t grid = int64_t(per_sm) * sms;
  const int64_t want = (warps_needed + 7) / 8;
  if (want < grid) grid = want;
  if (a.grid_cap > 0 && grid > a.grid_cap) grid = a.grid_cap;
  if (grid < 1) grid = 1;
  if (grid_out) *grid_out = int(grid);
  // Cooperative attribute through cudaLaunchKernelEx: co-residency is guaranteed (the grid
  // barrier relies on it) and the launch can be captured into a CUDA graph.
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(grid));
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = lpa_dynamic_smem(mode, a.wt == nullptr, a.stage != 0);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void *args[] = {const_cast<LpaArgs *>(&a)};
  return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace rak
