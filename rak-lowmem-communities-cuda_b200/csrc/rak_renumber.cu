// rak_renumber.cu -- a copy of a resident graph renumbered in its plan's work order.
//
// The plan sorts vertices heaviest first (split vertices, lane groups G = 32 .. 2, then one-lane
// vertices by descending degree). Renumbering vertex order[i] as i gives a CSR whose work order is
// the identity: the per-vertex reads of a run (work-order entry, flag, offsets, own label) become
// consecutive, consecutive one-lane vertices have adjacent edge lists, and the labels and flags of
// the highest-degree vertices -- the ones most edges point to -- share cache lines instead of
// sitting one per line across the whole label array. Labels keep their values: a vertex starts
// with its original id (or its caller-given initial label), so the pickless rule compares the same
// numbers as on the graph as given, and the result is gathered back into the original numbering.
//
// The reference does the same kind of thing on the host: it rebuilds its CSR in the order of its
// degree partition before the upload (inc/rakLowmemCuda.hxx:505-519, 563-568).
#include <cstdint>

#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include "rak_internal.hpp"

namespace rak {
namespace {

constexpr int TPB = 256;

inline int grid_of(int64_t items, int per_thread) {
  int64_t g = (items + int64_t(TPB) * per_thread - 1) / (int64_t(TPB) * per_thread);
  if (g < 1) g = 1;
  if (g > 148 * 64) g = 148 * 64;
  return int(g);
}

__global__ void k_rn_inverse(const uint32_t *__restrict__ order, int64_t n, uint32_t *__restrict__ inv) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = tid; i < n; i += nt) inv[__ldg(order + i)] = uint32_t(i);
}

// Degrees in the new numbering; entry n is 0, so an exclusive scan of n+1 entries gives the offsets.
template <class O>
__global__ void k_rn_degrees(const O *__restrict__ off, const uint32_t *__restrict__ order, int64_t n,
                             O *__restrict__ deg) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = tid; i <= n; i += nt) {
    if (i == n) { deg[i] = O(0); continue; }
    const uint32_t u = __ldg(order + i);
    deg[i] = O(__ldg(off + u + 1) - __ldg(off + u));
  }
}

// Rows [0, split) -- the vertices above the one-lane degree limit -- one warp per row, lanes
// striding over its edges; rows [split, n) one thread per row. Targets are renumbered, weights and
// the edge order within each row are kept.
template <class O>
__global__ void k_rn_edges(const O *__restrict__ off, const uint32_t *__restrict__ tgt, const float *__restrict__ wt,
                           const uint32_t *__restrict__ order, const uint32_t *__restrict__ inv,
                           const O *__restrict__ noff, int64_t n, int64_t split, uint32_t *__restrict__ ntgt,
                           float *__restrict__ nwt) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (int64_t i = tid >> 5; i < split; i += nt >> 5) {
    const uint32_t u = __ldg(order + i);
    const int64_t eb = int64_t(__ldg(off + u)), ee = int64_t(__ldg(off + u + 1)), db = int64_t(__ldg(noff + i));
    for (int64_t e = eb + lane; e < ee; e += 32) {
      ntgt[db + (e - eb)] = __ldg(inv + __ldg(tgt + e));
      if (wt) nwt[db + (e - eb)] = __ldg(wt + e);
    }
  }
  for (int64_t i = split + tid; i < n; i += nt) {
    const uint32_t u = __ldg(order + i);
    const int64_t eb = int64_t(__ldg(off + u)), ee = int64_t(__ldg(off + u + 1)), db = int64_t(__ldg(noff + i));
    for (int64_t e = eb; e < ee; ++e) {
      ntgt[db + (e - eb)] = __ldg(inv + __ldg(tgt + e));
      if (wt) nwt[db + (e - eb)] = __ldg(wt + e);
    }
  }
}

__global__ void k_rn_iota(uint32_t *__restrict__ p, int64_t n) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = tid; i < n; i += nt) p[i] = uint32_t(i);
}

// Labels and flags of a run in the new numbering: new vertex i is order[i] of the graph as given.
// pos (runs labelled by the reference order): a label is the position of that vertex id in it.
__global__ void k_rn_init(const uint32_t *__restrict__ order, const uint32_t *__restrict__ q,
                          const uint32_t *__restrict__ pos, const uint8_t *__restrict__ flags, int64_t n,
                          uint32_t *__restrict__ lab, uint8_t *__restrict__ aff) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = tid; i < n; i += nt) {
    const uint32_t u = __ldg(order + i);
    const uint32_t c = q ? __ldg(q + u) : u;
    lab[i] = pos ? __ldg(pos + c) : c;
    aff[i] = flags ? uint8_t(__ldg(flags + u) != 0) : uint8_t(1);
  }
}

__global__ void k_rn_gather(const uint32_t *__restrict__ lab, const uint32_t *__restrict__ inv, int64_t n,
                            uint32_t *__restrict__ out) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t v = tid; v < n; v += nt) out[v] = __ldg(lab + __ldg(inv + v));
}

template <class O>
cudaError_t renumber_t(const O *off, const uint32_t *tgt, const float *wt, const uint32_t *order, int64_t n,
                       int64_t split, uint32_t *inv, O *deg, O *noff, uint32_t *ntgt, float *nwt, uint32_t *ident,
                       void *temp, size_t *temp_bytes, cudaStream_t st) {
  size_t need = 0;
  cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, need, deg, noff, n + 1, st);
  if (e != cudaSuccess) return e;
  if (!temp) { *temp_bytes = need; return cudaSuccess; }
  if (*temp_bytes < need) return cudaErrorInvalidValue;
  k_rn_inverse<<<grid_of(n, 4), TPB, 0, st>>>(order, n, inv);
  k_rn_degrees<O><<<grid_of(n + 1, 4), TPB, 0, st>>>(off, order, n, deg);
  if ((e = cub::DeviceScan::ExclusiveSum(temp, need, deg, noff, n + 1, st)) != cudaSuccess) return e;
  k_rn_edges<O><<<148 * 8, TPB, 0, st>>>(off, tgt, wt, order, inv, noff, n, split, ntgt, nwt);
  k_rn_iota<<<grid_of(n, 4), TPB, 0, st>>>(ident, n);
  return cudaGetLastError();
}

}  // namespace

cudaError_t renumber_graph(const void *off, bool off64, const uint32_t *tgt, const float *wt, const uint32_t *order,
                           int64_t n, int64_t split, uint32_t *inv, void *deg, void *noff, uint32_t *ntgt, float *nwt,
                           uint32_t *ident, void *temp, size_t *temp_bytes, cudaStream_t st) {
  if (off64)
    return renumber_t<int64_t>(static_cast<const int64_t *>(off), tgt, wt, order, n, split, inv,
                               static_cast<int64_t *>(deg), static_cast<int64_t *>(noff), ntgt, nwt, ident, temp,
                               temp_bytes, st);
  return renumber_t<int32_t>(static_cast<const int32_t *>(off), tgt, wt, order, n, split, inv,
                             static_cast<int32_t *>(deg), static_cast<int32_t *>(noff), ntgt, nwt, ident, temp,
                             temp_bytes, st);
}

cudaError_t launch_renumbered_init(const uint32_t *order, const uint32_t *q, const uint32_t *pos, const uint8_t *flags,
                                   int64_t n, uint32_t *lab, uint8_t *aff, cudaStream_t st) {
  k_rn_init<<<grid_of(n, 4), TPB, 0, st>>>(order, q, pos, flags, n, lab, aff);
  return cudaGetLastError();
}

cudaError_t launch_renumbered_gather(const uint32_t *lab, const uint32_t *inv, int64_t n, uint32_t *out,
                                     cudaStream_t st) {
  k_rn_gather<<<grid_of(n, 4), TPB, 0, st>>>(lab, inv, n, out);
  return cudaGetLastError();
}

}  // namespace rak
