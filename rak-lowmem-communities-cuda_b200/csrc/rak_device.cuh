// rak_device.cuh -- device primitives: the per-lane weighted Misra-Gries / Boyer-Moore sketch held
// in registers, lane-tree merges over warp shuffles, and a bounded grid barrier.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "rak_hash.hpp"

namespace rak {

constexpr uint32_t NONE = 0xFFFFFFFFu;  // sketch key that matches no community
constexpr unsigned FULL = 0xFFFFFFFFu;

// A sketch of S (key, weight) slots in registers. S == 1 is the Boyer-Moore vote.
template <int S>
struct Sketch {
  uint32_t k[S];
  float w[S];
};

// The two rule sets of the reference: its CPU code's (inc/rakLowmem.hxx) and its GPU code's
// (inc/sketchCuda.hxx, inc/rakLowmemCuda.hxx). They differ in which free slot a new key takes,
// whether decrements clamp at zero, how the argmax breaks ties, the Boyer-Moore starting candidate
// and the weight test of the move rule. The synchronous exact mode follows the CPU rules (bit-exact
// against the reference CPU code); the other modes run either set, chosen per launch (the CPU rules
// by default: under the GPU rules' unclamped decrement R-MAT-like graphs collapse into one
// community, as they do on the reference GPU path).
enum : int { RULE_CPU = 1, RULE_GPU = 2 };

// Cleared sketch. Boyer-Moore under the GPU rules starts from the vertex's own label d with weight
// 0 (inc/rakLowmemCuda.hxx:41-43); otherwise keys start as NONE.
template <int S, int RULE = RULE_CPU>
__device__ __forceinline__ void sk_clear(Sketch<S> &s, uint32_t d = NONE) {
#pragma unroll
  for (int i = 0; i < S; ++i) { s.k[i] = NONE; s.w[i] = 0.0f; }
  if constexpr (S == 1 && RULE == RULE_GPU) s.k[0] = d;
}

// Weighted Misra-Gries accumulate with the reference CPU rule (inc/rakLowmem.hxx:63-89): add x to
// every slot keyed c; otherwise the LAST zero-weight slot takes (c, x); otherwise every weight
// drops by x, clamped at zero. Only adds, subtracts and max: bit-identical to the CPU.
// Hits (the common case once labels settle) leave early; the miss path runs only when needed.
#ifndef RAK_MG_MINFIRST
#define RAK_MG_MINFIRST 0
#endif
template <int S>
__device__ __forceinline__ void mg_acc(Sketch<S> &s, uint32_t c, float x) {
  bool hit = false;
#pragma unroll
  for (int i = 0; i < S; ++i)
    if (s.k[i] == c) { s.w[i] = __fadd_rn(s.w[i], x); hit = true; }
  if (hit) return;
#if RAK_MG_MINFIRST
  // every weight positive: no free slot, the decrement follows (same outcome as the search below)
  float mn = s.w[0];
#pragma unroll
  for (int i = 1; i < S; ++i) mn = fminf(mn, s.w[i]);
  if (mn > 0.0f) {
#pragma unroll
    for (int i = 0; i < S; ++i) s.w[i] = fmaxf(__fsub_rn(s.w[i], x), 0.0f);
    return;
  }
#endif
  int f = -1;
#pragma unroll
  for (int i = 0; i < S; ++i)
    if (s.w[i] == 0.0f) f = i;
  if (f >= 0) {
#pragma unroll
    for (int i = 0; i < S; ++i)
      if (i == f) { s.k[i] = c; s.w[i] = x; }
  } else {
#pragma unroll
    for (int i = 0; i < S; ++i) s.w[i] = fmaxf(__fsub_rn(s.w[i], x), 0.0f);
  }
}

// Weighted Misra-Gries accumulate with the reference GPU rule (inc/sketchCuda.hxx:73-108, one
// thread's view of sketchAccumulateWarpCudU): add x to every slot keyed c; otherwise the FIRST slot
// whose weight is exactly zero takes (c, x); otherwise every weight drops by x, with no clamp
// (weights may go negative; a negative slot is not free).
template <int S>
__device__ __forceinline__ void mg_acc_gpu(Sketch<S> &s, uint32_t c, float x) {
  bool hit = false;
#pragma unroll
  for (int i = 0; i < S; ++i)
    if (s.k[i] == c) { s.w[i] = __fadd_rn(s.w[i], x); hit = true; }
  if (hit) return;
  int f = S;
#pragma unroll
  for (int i = S - 1; i >= 0; --i)
    if (s.w[i] == 0.0f) f = i;
  if (f < S) {
#pragma unroll
    for (int i = 0; i < S; ++i)
      if (i == f) { s.k[i] = c; s.w[i] = x; }
  } else {
#pragma unroll
    for (int i = 0; i < S; ++i) s.w[i] = __fsub_rn(s.w[i], x);
  }
}

// Weighted Boyer-Moore vote (inc/rakLowmem.hxx:120-126, inc/rakLowmemCuda.hxx:49-51; the same
// arithmetic under both rule sets).
__device__ __forceinline__ void bm_acc(Sketch<1> &s, uint32_t c, float x) {
  if (c == s.k[0]) s.w[0] = __fadd_rn(s.w[0], x);
  else if (s.w[0] > x) s.w[0] = __fsub_rn(s.w[0], x);
  else { s.k[0] = c; s.w[0] = x; }
}

template <int S, int RULE = RULE_CPU>
__device__ __forceinline__ void sk_acc(Sketch<S> &s, uint32_t c, float x) {
  if constexpr (S == 1) bm_acc(s, c, x);
  else if constexpr (RULE == RULE_GPU) mg_acc_gpu(s, c, x);
  else mg_acc(s, c, x);
}

// Merge by re-accumulating the other sketch's non-zero slots in slot order
// (inc/sketchCuda.hxx:150-158).
template <int S, int RULE = RULE_CPU>
__device__ __forceinline__ void sk_merge(Sketch<S> &a, const uint32_t (&bk)[S], const float (&bw)[S]) {
#pragma unroll
  for (int j = 0; j < S; ++j)
    if (bw[j] != 0.0f) sk_acc<S, RULE>(a, bk[j], bw[j]);
}

// Fixed binary tree over the G lanes of each aligned lane group (G a power of two <= 32):
// at each level lane s < off merges the sketch of lane s+off. The group's result is in its
// lane 0. Every lane of the warp must call this with the same G.
template <int S, int RULE = RULE_CPU>
__device__ __forceinline__ void sk_tree(Sketch<S> &s, int G) {
  for (int off = G >> 1; off >= 1; off >>= 1) {
    uint32_t bk[S];
    float bw[S];
#pragma unroll
    for (int j = 0; j < S; ++j) {
      bk[j] = __shfl_down_sync(FULL, s.k[j], off, G);
      bw[j] = __shfl_down_sync(FULL, s.w[j], off, G);
    }
    sk_merge<S, RULE>(s, bk, bw);
  }
}

// CPU rule: linear argmax with strict '>' from weight 0 (inc/rakLowmem.hxx:164-171).
// GPU rule: the tournament of sketchMaxGroupReduceCudU (inc/sketchCuda.hxx:190-201) -- at each
// level slot i takes slot i+S/2 only if strictly heavier -- whose winner may weigh <= 0.
template <int S, int RULE = RULE_CPU>
__device__ __forceinline__ void sk_choose(const Sketch<S> &s, uint32_t &c, float &w) {
  if constexpr (RULE == RULE_GPU) {
    uint32_t k[S];
    float x[S];
#pragma unroll
    for (int i = 0; i < S; ++i) { k[i] = s.k[i]; x[i] = s.w[i]; }
#pragma unroll
    for (int ds = S / 2; ds >= 1; ds /= 2) {
#pragma unroll
      for (int i = 0; i < ds; ++i)
        if (x[i + ds] > x[i]) { k[i] = k[i + ds]; x[i] = x[i + ds]; }
    }
    c = k[0];
    w = x[0];
  } else {
    c = NONE;
    w = 0.0f;
#pragma unroll
    for (int i = 0; i < S; ++i)
      if (s.w[i] > w) { w = s.w[i]; c = s.k[i]; }
  }
}

// Tie rule of hashed ties: the CPU rules' argmax (largest weight) except that a maximum shared by
// several slots goes to the key with the largest tie_hash(u, key, l) -- a fixed pseudo-random order
// per vertex and iteration, so no neighbour position is preferred the way "most recently inserted"
// prefers the last neighbour in edge order (on grids: one direction). Ties between equal hashes keep
// the lower slot.
__host__ __device__ __forceinline__ uint64_t tie_hash(uint32_t u, uint32_t key, uint32_t l) {
  return mix64((uint64_t(key) << 32 | uint64_t(u)) ^ (uint64_t(l) * 0xD6E8FEB86659FD93ull));
}
template <int S>
__device__ __forceinline__ void sk_choose_hashed(const Sketch<S> &s, uint32_t u, uint32_t l, uint32_t &c, float &w) {
  c = NONE;
  w = 0.0f;
  uint64_t hb = 0;
#pragma unroll
  for (int i = 0; i < S; ++i) {
    const uint64_t h = tie_hash(u, s.k[i], l);
    if (s.w[i] > w || (s.w[i] == w && w > 0.0f && h > hb)) { w = s.w[i]; c = s.k[i]; hb = h; }
  }
}

// ---- run-wide state shared by all blocks of a persistent launch -------------------------
struct RunState {
  unsigned int bar;         // grid barrier arrivals (monotone within a launch)
  unsigned int abort;       // set when any wait gives up
  unsigned int error;       // rak_status of the failure
  unsigned int iterations;  // iterations performed
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier for a co-resident (cooperative) launch. Arrival counts are monotone, so
// barrier number `epoch` (1-based) completes when bar >= epoch * gridDim.x. The wait is bounded
// by timeout_ns of wall time; on expiry it records RAK_ERR_TIMEOUT (5), raises abort and every
// block leaves. Returns false when the launch must stop.
__device__ __forceinline__ bool grid_barrier(RunState *rs, unsigned int epoch, long long timeout_ns) {
  __shared__ unsigned int stop;
  __syncthreads();
  if (threadIdx.x == 0) {
    stop = 0;
    __threadfence();
    atomicAdd(&rs->bar, 1u);
    const unsigned int target = epoch * gridDim.x;
    const unsigned long long t0 = global_ns();
    unsigned int ns = 32;
    while (ld_acquire(&rs->bar) < target) {
      if (*(volatile unsigned int *)&rs->abort) { stop = 1; break; }
      if ((long long)(global_ns() - t0) > timeout_ns) {
        atomicCAS(&rs->error, 0u, 5u);
        atomicExch(&rs->abort, 1u);
        stop = 1;
        break;
      }
      __nanosleep(ns);
      if (ns < 1024) ns <<= 1;
    }
    __threadfence();
  }
  __syncthreads();
  return stop == 0;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

}  // namespace rak
