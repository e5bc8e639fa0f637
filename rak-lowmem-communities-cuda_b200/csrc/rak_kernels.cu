// rak_kernels.cu -- plan building, validation, initialisation and FP64 modularity kernels.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "rak_device.cuh"
#include "rak_internal.hpp"

namespace rak {

namespace {

constexpr int TPB = 256;

inline int grid_for(int64_t n, int per_thread = 1) {
  int64_t g = (n + int64_t(TPB) * per_thread - 1) / (int64_t(TPB) * per_thread);
  if (g < 1) g = 1;
  if (g > 148 * 64) g = 148 * 64;
  return int(g);
}

// CSR rules: offsets[0] == 0, non-decreasing, offsets[n] == m, every target < n.
// Any violation sets *bad to 1 (a missing offset property) or 2 (a target out of range).
template <class O>
__global__ void k_validate(const O *off, const uint32_t *tgt, int64_t n, int64_t m, unsigned int *bad) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t u = tid; u < n; u += nt) {
    const int64_t a = int64_t(off[u]), b = int64_t(off[u + 1]);
    if (a > b || a < 0 || b > m) atomicOr(bad, 1u);
  }
  if (tid == 0 && (int64_t(off[0]) != 0 || int64_t(off[n]) != m)) atomicOr(bad, 1u);
  for (int64_t e = tid; e < m; e += nt)
    if (int64_t(tgt[e]) >= n) atomicOr(bad, 2u);
}

// Plan sort key of every vertex (plan_key) and a histogram of keys.
template <class O>
__global__ void k_plan_keys(const O *off, int64_t n, Layout ly, uint32_t *keys, uint32_t *vids,
                            unsigned long long *hist, int nkeys) {
  extern __shared__ unsigned int sh[];
  for (int i = threadIdx.x; i < nkeys; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t u = tid; u < n; u += nt) {
    const uint32_t k = plan_key(int64_t(off[u + 1]) - int64_t(off[u]), ly);
    keys[u] = k;
    vids[u] = uint32_t(u);
    atomicAdd(&sh[k], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nkeys; i += blockDim.x)
    if (sh[i]) atomicAdd(hist + i, (unsigned long long)sh[i]);
}

template <class O>
__global__ void k_hub_degrees(const O *off, const uint32_t *order, int64_t nhub, int64_t *deg) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t h = tid; h < nhub; h += nt) {
    const uint32_t u = order[h];
    deg[h] = int64_t(off[u + 1]) - int64_t(off[u]);
  }
}

__global__ void k_init_labels(uint32_t *v0, uint32_t *v1, const uint32_t *q, int64_t n) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t u = tid; u < n; u += nt) {
    const uint32_t c = q ? q[u] : uint32_t(u);
    v0[u] = c;
    if (v1) v1[u] = c;
  }
}

// Labels as positions in the reference's vertex order: v[u] = pos[q ? q[u] : u].
__global__ void k_init_labels_mapped(uint32_t *v0, const uint32_t *q, const uint32_t *pos, int64_t n) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t u = tid; u < n; u += nt) v0[u] = __ldg(pos + (q ? q[u] : uint32_t(u)));
}

// Positions back to vertex ids: m[u] = ks[m[u]].
__global__ void k_labels_to_ids(uint32_t *m, const uint32_t *ks, int64_t n) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t u = tid; u < n; u += nt) m[u] = __ldg(ks + m[u]);
}

// The reference GPU path's vertex order, per segment (one graph of a batch, or the whole graph):
// vertex ids in order, partitioned by degree < 4, then the rest by degree < 128, each pass with the
// two-pointer exchange of libstdc++'s std::partition. For a pass over the range [lo, e) of a
// segment with c matching elements: the k-th non-matching element left of lo + c (a hole, ranked
// from the left) swaps with the k-th matching element from lo + c on (a mover, ranked from the
// right). Ranks come from one exclusive prefix count P of the match flags over all segments; flags
// are 0 left of lo, so P[i] - P[b] counts the matches in [lo, i).
struct Seg {
  int64_t b, e;
  uint32_t g;
};
__device__ __forceinline__ Seg seg_of(const uint32_t *gid, const int64_t *vbase, int64_t n, int64_t i) {
  if (!gid) return {0, n, 0u};
  const uint32_t g = gid[i];
  return {vbase[g], vbase[g + 1], g};
}

template <class O>
__global__ void k_ro_flags(const O *off, const uint32_t *ks, int64_t n, const uint32_t *gid, const int64_t *vbase,
                           const uint32_t *lo_cnt, int64_t limit, uint32_t *f) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = tid; i <= n; i += nt) {
    if (i == n) { f[n] = 0u; continue; }
    const Seg s = seg_of(gid, vbase, n, i);
    const int64_t lo = s.b + (lo_cnt ? lo_cnt[s.g] : 0u);
    const uint32_t v = ks[i];
    f[i] = i >= lo && int64_t(off[v + 1]) - int64_t(off[v]) < limit ? 1u : 0u;
  }
}

// Matches per segment: cnt[g] = P[e] - P[b].
__global__ void k_ro_count(const uint32_t *P, const int64_t *vbase, int64_t ngraphs, int64_t n, uint32_t *cnt) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t g = tid; g < ngraphs; g += nt) {
    const int64_t b = vbase ? vbase[g] : 0, e = vbase ? vbase[g + 1] : n;
    cnt[g] = P[e] - P[b];
  }
}

__global__ void k_ro_movers(const uint32_t *f, const uint32_t *P, int64_t n, const uint32_t *gid, const int64_t *vbase,
                            const uint32_t *lo_cnt, const uint32_t *cnt, uint32_t *mover) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = tid; i < n; i += nt) {
    if (!f[i]) continue;
    const Seg s = seg_of(gid, vbase, n, i);
    const int64_t lo = s.b + (lo_cnt ? lo_cnt[s.g] : 0u), c = cnt[s.g];
    const int64_t pp = int64_t(P[i]) - int64_t(P[s.b]);
    if (i - lo >= c) mover[lo + (c - pp - 1)] = uint32_t(i - s.b);
  }
}

__global__ void k_ro_swap(const uint32_t *f, const uint32_t *P, int64_t n, const uint32_t *gid, const int64_t *vbase,
                          const uint32_t *lo_cnt, const uint32_t *cnt, const uint32_t *mover, uint32_t *ks) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = tid; i < n; i += nt) {
    if (f[i]) continue;
    const Seg s = seg_of(gid, vbase, n, i);
    const int64_t lo = s.b + (lo_cnt ? lo_cnt[s.g] : 0u), c = cnt[s.g];
    if (i < lo || i - lo >= c) continue;
    const int64_t pp = int64_t(P[i]) - int64_t(P[s.b]);
    const int64_t j = s.b + mover[lo + (i - lo - pp)];
    const uint32_t t = ks[i];
    ks[i] = ks[j];
    ks[j] = t;
  }
}

__global__ void k_iota(uint32_t *a, int64_t n) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = tid; i < n; i += nt) a[i] = uint32_t(i);
}

__global__ void k_inverse(const uint32_t *ks, uint32_t *pos, int64_t n) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = tid; i < n; i += nt) pos[ks[i]] = uint32_t(i);
}

__global__ void k_init_flags(uint8_t *f0, uint8_t *f1, const uint8_t *f, int64_t n) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t u = tid; u < n; u += nt) {
    f0[u] = f ? (f[u] ? 1 : 0) : 1;
    if (f1) f1[u] = 0;
  }
}

// FP64 modularity terms (inc/properties.hxx:177-192): per vertex u with community c, the weight
// of edges to its own community (summed into sums[0]), its total weight (into ctot[c]) and the
// grand total (sums[1] = 2M). A second kernel sums ctot[c]^2 into sums[2].
template <class O>
__global__ void k_mod_vertex(const O *off, const uint32_t *tgt, const float *wt, int64_t n,
                             const uint32_t *labels, double *ctot, double *sums) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5, nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  double in_acc = 0.0, tot_acc = 0.0;
  for (int64_t u = w0; u < n; u += nw) {  // one warp per vertex
    const uint32_t c = labels[u];
    if (int64_t(c) >= n) {  // not a vertex id: counted, and the host reports the error
      if (lane == 0) atomicAdd(sums + 3, 1.0);
      continue;
    }
    const int64_t eb = int64_t(off[u]), ee = int64_t(off[u + 1]);
    double kin = 0.0, kt = 0.0;
    for (int64_t e = eb + lane; e < ee; e += 32) {
      const double w = wt ? double(wt[e]) : 1.0;
      kt += w;
      if (labels[tgt[e]] == c) kin += w;
    }
    kin = warp_sum(kin);
    kt = warp_sum(kt);
    if (lane == 0 && kt != 0.0) atomicAdd(ctot + c, kt);
    in_acc += kin;
    tot_acc += kt;
  }
  __shared__ double s_in[TPB / 32], s_tot[TPB / 32];
  if (lane == 0) { s_in[threadIdx.x >> 5] = in_acc; s_tot[threadIdx.x >> 5] = tot_acc; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < TPB / 32; ++i) { a += s_in[i]; b += s_tot[i]; }
    atomicAdd(sums + 0, a);
    atomicAdd(sums + 1, b);
  }
}

__global__ void k_mod_square(const double *ctot, int64_t n, double *sums) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  double acc = 0.0;
  for (int64_t c = tid; c < n; c += nt) acc += ctot[c] * ctot[c];
  acc = warp_sum(acc);
  __shared__ double s[TPB / 32];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int i = 0; i < TPB / 32; ++i) a += s[i];
    atomicAdd(sums + 2, a);
  }
}

// ---- batches of graphs ------------------------------------------------------------------------
// gid[u] = graph of vertex u, from the graph vertex offsets.
__global__ void k_batch_gid(const int64_t *vbase, int64_t ngraphs, int64_t n, uint32_t *gid) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t u = tid; u < n; u += nt) {  // the last g with vbase[g] <= u: binary search
    int64_t lo = 0, hi = ngraphs;          // vbase[lo] <= u < vbase[hi]
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (vbase[mid] <= u) lo = mid;
      else hi = mid;
    }
    gid[u] = uint32_t(lo);
  }
}

// Batch CSR rules: graph offsets non-decreasing from 0 to n, and every target (a local id) below
// its own graph's vertex count. Violations set *bad.
__global__ void k_batch_validate(const int64_t *vbase, int64_t ngraphs, int64_t n, const int64_t *off,
                                 const uint32_t *tgt, const uint32_t *gid, unsigned int *bad) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  if (tid == 0 && (vbase[0] != 0 || vbase[ngraphs] != n)) atomicOr(bad, 1u);
  for (int64_t g = tid; g < ngraphs; g += nt)
    if (vbase[g] > vbase[g + 1]) atomicOr(bad, 1u);
  for (int64_t u = tid; u < n; u += nt) {
    const uint32_t g = gid[u];
    const int64_t ng = vbase[g + 1] - vbase[g];
    for (int64_t e = off[u]; e < off[u + 1]; ++e)
      if (int64_t(tgt[e]) >= ng) { atomicOr(bad, 2u); break; }
  }
}

// Labels at the start of a batch run: global vertex ids, from local initial labels q if given.
__global__ void k_batch_init(uint32_t *v0, uint32_t *v1, const uint32_t *q, const uint32_t *gid,
                             const int64_t *vbase, int64_t n) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t u = tid; u < n; u += nt) {
    const uint32_t c = q ? uint32_t(vbase[gid[u]]) + q[u] : uint32_t(u);
    v0[u] = c;
    if (v1) v1[u] = c;
  }
}

// Labels of an asynchronous batch run in the reference order: global position of the (local)
// initial label within its graph's order.
__global__ void k_batch_init_mapped(uint32_t *v0, const uint32_t *q, const uint32_t *gid, const int64_t *vbase,
                                    const uint32_t *pos, int64_t n) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t u = tid; u < n; u += nt) v0[u] = __ldg(pos + (q ? uint32_t(vbase[gid[u]]) + q[u] : uint32_t(u)));
}

// Global positions back to local vertex ids.
__global__ void k_batch_finish_mapped(const uint32_t *v0, const uint32_t *ks, const uint32_t *gid,
                                      const int64_t *vbase, int64_t n, uint32_t *membership) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t u = tid; u < n; u += nt) membership[u] = __ldg(ks + v0[u]) - uint32_t(vbase[gid[u]]);
}

// Final local labels: the buffer the last iteration wrote (decided on the device from the
// iteration count, so the launch sequence needs no host round trip), minus the graph's offset.
__global__ void k_batch_finish(const uint32_t *v0, const uint32_t *v1, const RunState *rs, const uint32_t *gid,
                               const int64_t *vbase, int64_t n, uint32_t *membership) {
  const uint32_t *src = (v1 && (rs->iterations & 1u)) ? v1 : v0;
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t u = tid; u < n; u += nt) membership[u] = src[u] - uint32_t(vbase[gid[u]]);
}

// Per-graph FP64 modularity terms: internal weight and total weight per graph, community totals
// per global label (ctot), then squared community totals per graph. labels are local.
__global__ void k_batch_mod_vertex(const int64_t *off, const uint32_t *tgt, const float *wt, const uint32_t *gid,
                                   const int64_t *vbase, int64_t n, const uint32_t *labels, double *ctot,
                                   double *gin, double *gtot, double *bad) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5, nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t u = w0; u < n; u += nw) {
    const uint32_t g = gid[u];
    const int64_t base = vbase[g], ng = vbase[g + 1] - base;
    const uint32_t c = labels[u];
    if (int64_t(c) >= ng) {
      if (lane == 0) atomicAdd(bad, 1.0);
      continue;
    }
    double kin = 0.0, kt = 0.0;
    for (int64_t e = off[u] + lane; e < off[u + 1]; e += 32) {
      const double w = wt ? double(wt[e]) : 1.0;
      kt += w;
      if (labels[base + tgt[e]] == c) kin += w;
    }
    kin = warp_sum(kin);
    kt = warp_sum(kt);
    if (lane == 0 && kt != 0.0) {
      atomicAdd(ctot + base + c, kt);
      atomicAdd(gin + g, kin);
      atomicAdd(gtot + g, kt);
    }
  }
}

__global__ void k_batch_mod_square(const double *ctot, const uint32_t *gid, int64_t n, double *gsq) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t c = tid; c < n; c += nt)
    if (ctot[c] != 0.0) atomicAdd(gsq + gid[c], ctot[c] * ctot[c]);
}

__global__ void k_fill_f32(float *p, int64_t count, float v) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = tid; i < count; i += nt) p[i] = v;
}

// Packs graphs into a batch CSR: graph blockIdx.y's offsets rebased by its first edge slot, its
// targets copied, its weights copied (or 1.0 where the batch is weighted and the graph is not);
// an item without targets has its edges in place already (only the offsets are rebased). The CSR
// rules are checked on the way (bad[y]: 1 = offsets, 2 = a target out of range); the copies touch
// only the n + 1 offsets and m edges the graph declares.
__global__ void k_gather_graphs(const GatherItem *items, int64_t *off_dst, uint32_t *tgt_dst, float *wt_dst,
                                unsigned int *bad) {
  const GatherItem it = items[blockIdx.y];
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  unsigned int b = 0;
  const int64_t *o64 = static_cast<const int64_t *>(it.off);
  const int32_t *o32 = static_cast<const int32_t *>(it.off);
  for (int64_t u = tid; u < it.n; u += nt) {
    const int64_t a = it.off64 ? o64[u] : int64_t(o32[u]);
    const int64_t z = it.off64 ? o64[u + 1] : int64_t(o32[u + 1]);
    off_dst[it.vdst + u] = a + it.edst;
    if (a > z) b |= 1u;
  }
  if (tid == 0) {
    const int64_t a = it.off64 ? o64[0] : int64_t(o32[0]);
    const int64_t z = it.off64 ? o64[it.n] : int64_t(o32[it.n]);
    if (a != 0 || z != it.m) b |= 1u;
  }
  const uint64_t lim = uint64_t(it.n);
  for (int64_t e = tid; it.tgt && e < it.m; e += nt) {
    const uint32_t t = it.tgt[e];
    tgt_dst[it.edst + e] = t;
    if (uint64_t(t) >= lim) b |= 2u;
    if (wt_dst) wt_dst[it.edst + e] = it.wt ? it.wt[e] : 1.0f;
  }
  if (b) atomicOr(bad + blockIdx.y, b);
}

}  // namespace

cudaError_t launch_fill_f32(float *p, int64_t count, float v, cudaStream_t st) {
  k_fill_f32<<<grid_for(count, 4), TPB, 0, st>>>(p, count, v);
  return cudaGetLastError();
}

cudaError_t launch_gather_graphs(const GatherItem *items, int count, int64_t max_elems, int64_t *off_dst,
                                 uint32_t *tgt_dst, float *wt_dst, unsigned int *bad, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  if (count > 65535) return cudaErrorInvalidValue;
  const int64_t bx = (max_elems + int64_t(TPB) * 8 - 1) / (int64_t(TPB) * 8);
  const dim3 grid(unsigned(bx < 1 ? 1 : (bx > 1024 ? 1024 : bx)), unsigned(count));
  k_gather_graphs<<<grid, TPB, 0, st>>>(items, off_dst, tgt_dst, wt_dst, bad);
  return cudaGetLastError();
}

cudaError_t launch_batch_gid(const int64_t *vbase, int64_t ngraphs, int64_t n, uint32_t *gid, cudaStream_t st) {
  k_batch_gid<<<grid_for(n, 4), TPB, 0, st>>>(vbase, ngraphs, n, gid);
  return cudaGetLastError();
}

cudaError_t launch_batch_validate(const int64_t *vbase, int64_t ngraphs, int64_t n, const int64_t *off,
                                  const uint32_t *tgt, const uint32_t *gid, unsigned int *bad, cudaStream_t st) {
  k_batch_validate<<<grid_for(n > ngraphs ? n : ngraphs, 4), TPB, 0, st>>>(vbase, ngraphs, n, off, tgt, gid, bad);
  return cudaGetLastError();
}

cudaError_t launch_batch_init(uint32_t *v0, uint32_t *v1, const uint32_t *q, const uint32_t *gid,
                              const int64_t *vbase, int64_t n, cudaStream_t st) {
  k_batch_init<<<grid_for(n, 4), TPB, 0, st>>>(v0, v1, q, gid, vbase, n);
  return cudaGetLastError();
}

cudaError_t launch_batch_init_mapped(uint32_t *v0, const uint32_t *q, const uint32_t *gid, const int64_t *vbase,
                                     const uint32_t *pos, int64_t n, cudaStream_t st) {
  k_batch_init_mapped<<<grid_for(n, 4), TPB, 0, st>>>(v0, q, gid, vbase, pos, n);
  return cudaGetLastError();
}

cudaError_t launch_batch_finish_mapped(const uint32_t *v0, const uint32_t *ks, const uint32_t *gid,
                                       const int64_t *vbase, int64_t n, uint32_t *membership, cudaStream_t st) {
  k_batch_finish_mapped<<<grid_for(n, 4), TPB, 0, st>>>(v0, ks, gid, vbase, n, membership);
  return cudaGetLastError();
}

cudaError_t launch_batch_finish(const uint32_t *v0, const uint32_t *v1, const void *rs, const uint32_t *gid,
                                const int64_t *vbase, int64_t n, uint32_t *membership, cudaStream_t st) {
  k_batch_finish<<<grid_for(n, 4), TPB, 0, st>>>(v0, v1, static_cast<const RunState *>(rs), gid, vbase, n, membership);
  return cudaGetLastError();
}

cudaError_t launch_batch_modularity(const int64_t *off, const uint32_t *tgt, const float *wt, const uint32_t *gid,
                                    const int64_t *vbase, int64_t n, const uint32_t *labels, double *ctot,
                                    double *gin, double *gtot, double *gsq, double *bad, cudaStream_t st) {
  k_batch_mod_vertex<<<grid_for(n * 32, 4), TPB, 0, st>>>(off, tgt, wt, gid, vbase, n, labels, ctot, gin, gtot, bad);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_batch_mod_square<<<grid_for(n, 4), TPB, 0, st>>>(ctot, gid, n, gsq);
  return cudaGetLastError();
}

cudaError_t launch_validate(const void *off, bool off64, const uint32_t *tgt, int64_t n, int64_t m,
                            unsigned int *bad, cudaStream_t st) {
  const int g = grid_for(n > m ? n : m, 4);
  if (off64) k_validate<int64_t><<<g, TPB, 0, st>>>(static_cast<const int64_t *>(off), tgt, n, m, bad);
  else k_validate<int32_t><<<g, TPB, 0, st>>>(static_cast<const int32_t *>(off), tgt, n, m, bad);
  return cudaGetLastError();
}

cudaError_t launch_plan_keys(const void *off, bool off64, int64_t n, Layout ly, uint32_t *keys,
                             uint32_t *vids, unsigned long long *hist, int nkeys, cudaStream_t st) {
  const int g = grid_for(n, 8);
  const size_t sh = size_t(nkeys) * sizeof(unsigned int);
  if (off64) k_plan_keys<int64_t><<<g, TPB, sh, st>>>(static_cast<const int64_t *>(off), n, ly, keys, vids, hist, nkeys);
  else k_plan_keys<int32_t><<<g, TPB, sh, st>>>(static_cast<const int32_t *>(off), n, ly, keys, vids, hist, nkeys);
  return cudaGetLastError();
}

// Stable radix sort of (key, vertex id) pairs: vertices grouped by region, ascending id within
// a key. With temp == nullptr only reports the temporary storage size.
cudaError_t plan_sort(uint32_t *keys_in, uint32_t *keys_out, uint32_t *vals_in, uint32_t *vals_out,
                      int64_t n, int end_bit, void *temp, size_t *temp_bytes, cudaStream_t st) {
  return cub::DeviceRadixSort::SortPairs(temp, *temp_bytes, keys_in, keys_out, vals_in, vals_out, n, 0,
                                         end_bit, st);
}

cudaError_t launch_hub_degrees(const void *off, bool off64, const uint32_t *order, int64_t nhub,
                               int64_t *deg, cudaStream_t st) {
  const int g = grid_for(nhub);
  if (off64) k_hub_degrees<int64_t><<<g, TPB, 0, st>>>(static_cast<const int64_t *>(off), order, nhub, deg);
  else k_hub_degrees<int32_t><<<g, TPB, 0, st>>>(static_cast<const int32_t *>(off), order, nhub, deg);
  return cudaGetLastError();
}

cudaError_t launch_init(uint32_t *vcom0, uint32_t *vcom1, const uint32_t *q, int64_t n, cudaStream_t st) {
  k_init_labels<<<grid_for(n, 4), TPB, 0, st>>>(vcom0, vcom1, q, n);
  return cudaGetLastError();
}

cudaError_t launch_init_mapped(uint32_t *vcom0, const uint32_t *q, const uint32_t *pos, int64_t n, cudaStream_t st) {
  k_init_labels_mapped<<<grid_for(n, 4), TPB, 0, st>>>(vcom0, q, pos, n);
  return cudaGetLastError();
}

cudaError_t launch_labels_to_ids(uint32_t *m, const uint32_t *ks, int64_t n, cudaStream_t st) {
  k_labels_to_ids<<<grid_for(n, 4), TPB, 0, st>>>(m, ks, n);
  return cudaGetLastError();
}

size_t ref_order_scratch_bytes(int64_t n, int64_t ngraphs) {
  size_t scan = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan, static_cast<const uint32_t *>(nullptr), static_cast<uint32_t *>(nullptr),
                                n + 1);
  const size_t arrays = size_t(n + 1) * 4 * 2 + size_t(n > 0 ? n : 1) * 4 + size_t(ngraphs > 0 ? ngraphs : 1) * 4 * 2;
  return ((arrays + 255) / 256) * 256 + ((scan + 255) / 256) * 256 + 256;
}

// The reference GPU path's vertex order (inc/rakLowmemCuda.hxx:505-519, 563) of every segment:
// gid/vbase describe a batch (ngraphs graphs; ks and pos then hold global vertex indices), or are
// null for one graph. ks[i] is the i-th vertex of that order, pos its inverse. No host round trip.
cudaError_t ref_order(const void *off, bool off64, int64_t n, const uint32_t *gid, const int64_t *vbase,
                      int64_t ngraphs, uint32_t *ks, uint32_t *pos, void *scratch, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (!gid) ngraphs = 1;
  uint8_t *p = static_cast<uint8_t *>(scratch);
  uint32_t *f = reinterpret_cast<uint32_t *>(p), *P = f + (n + 1), *mover = P + (n + 1);
  uint32_t *cnt1 = mover + n, *cnt2 = cnt1 + ngraphs;
  const size_t arrays = size_t(n + 1) * 4 * 2 + size_t(n) * 4 + size_t(ngraphs) * 4 * 2;
  void *cub_temp = p + ((arrays + 255) / 256) * 256;
  size_t cub_bytes = ref_order_scratch_bytes(n, ngraphs) - ((arrays + 255) / 256) * 256 - 256;
  k_iota<<<grid_for(n, 4), TPB, 0, st>>>(ks, n);
  for (int pass = 0; pass < 2; ++pass) {
    const uint32_t *lo_cnt = pass == 0 ? nullptr : cnt1;
    uint32_t *cnt = pass == 0 ? cnt1 : cnt2;
    const int64_t limit = pass == 0 ? 4 : 128;
    if (off64) k_ro_flags<int64_t><<<grid_for(n + 1, 4), TPB, 0, st>>>(static_cast<const int64_t *>(off), ks, n, gid, vbase, lo_cnt, limit, f);
    else k_ro_flags<int32_t><<<grid_for(n + 1, 4), TPB, 0, st>>>(static_cast<const int32_t *>(off), ks, n, gid, vbase, lo_cnt, limit, f);
    cudaError_t e = cub::DeviceScan::ExclusiveSum(cub_temp, cub_bytes, f, P, n + 1, st);
    if (e != cudaSuccess) return e;
    k_ro_count<<<grid_for(ngraphs, 1), TPB, 0, st>>>(P, gid ? vbase : nullptr, ngraphs, n, cnt);
    k_ro_movers<<<grid_for(n, 4), TPB, 0, st>>>(f, P, n, gid, vbase, lo_cnt, cnt, mover);
    k_ro_swap<<<grid_for(n, 4), TPB, 0, st>>>(f, P, n, gid, vbase, lo_cnt, cnt, mover, ks);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  k_inverse<<<grid_for(n, 4), TPB, 0, st>>>(ks, pos, n);
  return cudaGetLastError();
}

cudaError_t launch_init_flags(uint8_t *aff0, uint8_t *aff1, const uint8_t *f, int64_t n, cudaStream_t st) {
  k_init_flags<<<grid_for(n, 4), TPB, 0, st>>>(aff0, aff1, f, n);
  return cudaGetLastError();
}

// ctot: n doubles (zeroed by the caller), sums: 4 doubles (zeroed by the caller) receive
// [internal weight, total weight 2M, sum of squared community totals, labels >= n seen].
cudaError_t launch_modularity(const void *off, bool off64, const uint32_t *tgt, const float *wt, int64_t n,
                              const uint32_t *labels, double *ctot, double *sums, cudaStream_t st) {
  const int g = grid_for(n * 32, 4);
  if (off64) k_mod_vertex<int64_t><<<g, TPB, 0, st>>>(static_cast<const int64_t *>(off), tgt, wt, n, labels, ctot, sums);
  else k_mod_vertex<int32_t><<<g, TPB, 0, st>>>(static_cast<const int32_t *>(off), tgt, wt, n, labels, ctot, sums);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_mod_square<<<grid_for(n, 4), TPB, 0, st>>>(ctot, n, sums);
  return cudaGetLastError();
}

cudaError_t prepare_lpa(int slots, int mode, bool off64, bool unit, bool batch, bool stage) {
  const void *fn = nullptr;
  int per_sm = 0;
  switch (slots) {
    case 1: return resolve_lpa_slots<1>(mode, off64, unit, batch, stage, &fn, &per_sm);
    case 2: return resolve_lpa_slots<2>(mode, off64, unit, batch, stage, &fn, &per_sm);
    case 4: return resolve_lpa_slots<4>(mode, off64, unit, batch, stage, &fn, &per_sm);
    case 8: return resolve_lpa_slots<8>(mode, off64, unit, batch, stage, &fn, &per_sm);
    case 16: return resolve_lpa_slots<16>(mode, off64, unit, batch, stage, &fn, &per_sm);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_lpa(const LpaArgs &a, int slots, int mode, bool off64, cudaStream_t st, int *grid_out,
                       bool batch) {
  switch (slots) {
    case 1: return launch_lpa_slots<1>(a, mode, off64, batch, st, grid_out);
    case 2: return launch_lpa_slots<2>(a, mode, off64, batch, st, grid_out);
    case 4: return launch_lpa_slots<4>(a, mode, off64, batch, st, grid_out);
    case 8: return launch_lpa_slots<8>(a, mode, off64, batch, st, grid_out);
    case 16: return launch_lpa_slots<16>(a, mode, off64, batch, st, grid_out);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace rak
