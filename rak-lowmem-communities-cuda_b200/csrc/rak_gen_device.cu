// rak_gen_device.cu -- symmetric R-MAT and planted-partition SBM built on the device, bit-identical
// to the host generators (rak_gen.cpp, rak_gen_rmat and rak_gen_sbm): the same counter-based
// samples, both directions of every sample that is not a self-loop, adjacency sorted and
// duplicate-free, weights from the undirected pair's hash. A scale-27 graph (4.3 billion directed
// edges) takes seconds here instead of minutes on the host.
//
// Pipeline: one 64-bit key (u << bits | v) per direction of each sample (bits = scale for R-MAT, the
// bits of n - 1 for SBM; self-loops become an all-ones sentinel that sorts last) -> radix sort over
// 2*bits bits -> unique -> CSR from the run boundaries of u -> weights.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include "rak_hash.hpp"
#include "rak_internal.hpp"

namespace rak {
namespace {

constexpr int TPB = 256;
constexpr uint64_t STREAM_RMAT = 1, STREAM_WEIGHT = 2, STREAM_SBM = 3;  // as in rak_gen.cpp

inline unsigned grid_for(int64_t n) {
  int64_t b = (n + int64_t(TPB) * 4 - 1) / (int64_t(TPB) * 4);
  if (b < 1) b = 1;
  if (b > 148 * 64) b = 148 * 64;
  return unsigned(b);
}

// The host generator's sample i (rak_gen.cpp): each level takes 16 random bits; quadrant (0,0)
// with probability a, (0,1) b, (1,0) c, (1,1) d.
__device__ __forceinline__ void rmat_sample(int64_t i, int scale, uint64_t seed, uint32_t tA, uint32_t tAB,
                                            uint32_t tABC, uint32_t &u, uint32_t &v) {
  uint32_t uu = 0, vv = 0;
  uint64_t h = 0;
  for (int L = 0; L < scale; ++L) {
    if ((L & 3) == 0) h = rand64(seed, STREAM_RMAT, uint64_t(i) * 8 + uint64_t(L >> 2));
    const uint32_t r = uint32_t(h >> (16 * (L & 3))) & 0xFFFFu;
    const uint32_t ub = r >= tAB;
    const uint32_t vb = (r >= tA && r < tAB) || r >= tABC;
    uu = (uu << 1) | ub;
    vv = (vv << 1) | vb;
  }
  u = uu;
  v = vv;
}

__global__ void k_rmat_keys(int64_t samples, int scale, uint64_t seed, uint32_t tA, uint32_t tAB, uint32_t tABC,
                            uint64_t *keys) {
  const uint64_t sentinel = (uint64_t(1) << (2 * scale)) - 1;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < samples; i += int64_t(gridDim.x) * blockDim.x) {
    uint32_t u, v;
    rmat_sample(i, scale, seed, tA, tAB, tABC, u, v);
    const bool loop = u == v;
    keys[2 * i] = loop ? sentinel : (uint64_t(u) << scale | v);
    keys[2 * i + 1] = loop ? sentinel : (uint64_t(v) << scale | u);
  }
}

// The host generator's SBM sample i (rak_gen.cpp, rak_gen_sbm): u uniform; v inside u's block with
// probability fin (24-bit draw below fin24), else uniform outside it. Block b starts at
// ceil(b*n/k); the block of u is floor(u*k/n).
__device__ __forceinline__ uint32_t below_d(uint64_t h, uint64_t n) { return uint32_t(((h >> 32) * n) >> 32); }

__global__ void k_sbm_keys(int64_t samples, int64_t n, int64_t k, uint32_t fin24, uint64_t seed, int bits,
                           uint64_t *keys) {
  const uint64_t sentinel = (uint64_t(1) << (2 * bits)) - 1;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < samples; i += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t h0 = rand64(seed, STREAM_SBM, uint64_t(i) * 3);
    const uint64_t h1 = rand64(seed, STREAM_SBM, uint64_t(i) * 3 + 1);
    const uint64_t h2 = rand64(seed, STREAM_SBM, uint64_t(i) * 3 + 2);
    const uint32_t u = below_d(h0, uint64_t(n));
    const int64_t blk = int64_t(u) * k / n, lo = (blk * n + k - 1) / k, hi = ((blk + 1) * n + k - 1) / k;
    uint32_t v;
    if (uint32_t(h1 >> 40) < fin24 || hi - lo == n) {
      v = uint32_t(lo) + below_d(h2, uint64_t(hi - lo));
    } else {
      const uint32_t r = below_d(h2, uint64_t(n - (hi - lo)));
      v = r < uint32_t(lo) ? r : r + uint32_t(hi - lo);
    }
    const bool loop = u == v;
    keys[2 * i] = loop ? sentinel : (uint64_t(u) << bits | v);
    keys[2 * i + 1] = loop ? sentinel : (uint64_t(v) << bits | u);
  }
}

// CSR from the sorted unique keys: targets, and offsets filled at every change of u.
template <class O>
__global__ void k_keys_to_csr(const uint64_t *keys, int64_t m, int64_t n, int scale, O *off, uint32_t *tgt) {
  const uint64_t mask = (uint64_t(1) << scale) - 1;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t k = keys[i];
    const int64_t u = int64_t(k >> scale);
    tgt[i] = uint32_t(k & mask);
    const int64_t prev = i == 0 ? -1 : int64_t(keys[i - 1] >> scale);
    for (int64_t w = prev + 1; w <= u; ++w) off[w] = O(i);
    if (i == m - 1)
      for (int64_t w = u + 1; w <= n; ++w) off[w] = O(m);
  }
  if (m == 0)
    for (int64_t w = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; w <= n; w += int64_t(gridDim.x) * blockDim.x)
      off[w] = O(0);
}

// Symmetric weights in [lo, hi): one value per undirected pair from the pair's hash, rounded as
// the host computes it (a product, then a sum; no fused multiply-add).
__global__ void k_pair_weights(const uint64_t *keys, int64_t m, int scale, uint64_t seed, float lo, float span,
                               float *wt) {
  const uint64_t mask = (uint64_t(1) << scale) - 1;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t a = keys[i] >> scale, b = keys[i] & mask;
    const uint64_t key = a < b ? (a << 32 | b) : (b << 32 | a);
    wt[i] = __fadd_rn(lo, __fmul_rn(span, unit24(rand64(seed, STREAM_WEIGHT, key))));
  }
}

}  // namespace

namespace {

// The shared part of both generators: k0 holds nk keys over 2*bits bits (k1 the same size as
// scratch); sorts them, drops duplicates and the self-loop sentinel, builds the CSR of n vertices
// (weights from the pair hash when weighted) into out, and frees k0, k1.
cudaError_t build_from_keys(uint64_t *k0, uint64_t *k1, int64_t nk, int64_t n, int bits, uint64_t seed, bool weighted,
                            float w_lo, float w_hi, bool off64, cudaStream_t st, GenDeviceOut *out) {
  uint64_t *d_count = nullptr;
  void *temp = nullptr;
  cudaError_t e = cudaSuccess;
  auto fail = [&](cudaError_t err) {
    cudaFree(k0);
    cudaFree(k1);
    cudaFree(d_count);
    cudaFree(temp);
    cudaFree(out->offsets);
    cudaFree(out->targets);
    cudaFree(out->weights);
    *out = GenDeviceOut{};
    return err;
  };
  if ((e = cudaMalloc(&d_count, 8)) != cudaSuccess) return fail(e);
  cub::DoubleBuffer<uint64_t> db(k0, k1);
  size_t sort_bytes = 0, uniq_bytes = 0;
  if ((e = cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, db, nk, 0, 2 * bits, st)) != cudaSuccess) return fail(e);
  if ((e = cub::DeviceSelect::Unique(nullptr, uniq_bytes, db.Current(), db.Alternate(), d_count, nk, st)) !=
      cudaSuccess)
    return fail(e);
  if ((e = cudaMalloc(&temp, std::max<size_t>(std::max(sort_bytes, uniq_bytes), 16))) != cudaSuccess) return fail(e);
  if ((e = cub::DeviceRadixSort::SortKeys(temp, sort_bytes, db, nk, 0, 2 * bits, st)) != cudaSuccess) return fail(e);
  if ((e = cub::DeviceSelect::Unique(temp, uniq_bytes, db.Current(), db.Alternate(), d_count, nk, st)) != cudaSuccess)
    return fail(e);
  const uint64_t *uk = db.Alternate();
  int64_t count = 0;
  if ((e = cudaMemcpyAsync(&count, d_count, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return fail(e);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e);
  int64_t m = count;
  if (count > 0) {  // the sentinel, if any self-loop was drawn, is the last unique key
    uint64_t last = 0;
    if ((e = cudaMemcpy(&last, uk + count - 1, 8, cudaMemcpyDeviceToHost)) != cudaSuccess) return fail(e);
    if (last == (uint64_t(1) << (2 * bits)) - 1) --m;
  }
  if (!off64 && m >= (int64_t(1) << 31)) return fail(cudaErrorInvalidValue);
  if ((e = cudaMalloc(&out->offsets, size_t(n + 1) * (off64 ? 8 : 4))) != cudaSuccess) return fail(e);
  if ((e = cudaMalloc(&out->targets, size_t(std::max<int64_t>(m, 1)) * 4)) != cudaSuccess) return fail(e);
  if (weighted && (e = cudaMalloc(&out->weights, size_t(std::max<int64_t>(m, 1)) * 4)) != cudaSuccess) return fail(e);
  const unsigned g = grid_for(std::max(m, n + 1));
  if (off64) k_keys_to_csr<int64_t><<<g, TPB, 0, st>>>(uk, m, n, bits, static_cast<int64_t *>(out->offsets), out->targets);
  else k_keys_to_csr<int32_t><<<g, TPB, 0, st>>>(uk, m, n, bits, static_cast<int32_t *>(out->offsets), out->targets);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
  if (weighted) {
    k_pair_weights<<<grid_for(m), TPB, 0, st>>>(uk, m, bits, seed, w_lo, w_hi - w_lo, out->weights);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e);
  cudaFree(k0);
  cudaFree(k1);
  cudaFree(d_count);
  cudaFree(temp);
  out->n = n;
  out->m = m;
  out->peak_bytes = uint64_t(nk) * 16 + std::max(sort_bytes, uniq_bytes) + uint64_t(n + 1) * (off64 ? 8 : 4) +
                    uint64_t(m) * (weighted ? 8 : 4);
  return cudaSuccess;
}

cudaError_t alloc_keys(int64_t nk, uint64_t **k0, uint64_t **k1) {
  *k0 = *k1 = nullptr;
  cudaError_t e = cudaMalloc(k0, size_t(std::max<int64_t>(nk, 1)) * 8);
  if (e == cudaSuccess) e = cudaMalloc(k1, size_t(std::max<int64_t>(nk, 1)) * 8);
  if (e != cudaSuccess) {
    cudaFree(*k0);
    *k0 = nullptr;
  }
  return e;
}

}  // namespace

cudaError_t gen_rmat_device(int scale, int64_t samples, uint64_t seed, uint32_t tA, uint32_t tAB, uint32_t tABC,
                            bool weighted, float w_lo, float w_hi, bool off64, cudaStream_t st, GenDeviceOut *out) {
  *out = GenDeviceOut{};
  const int64_t nk = 2 * samples;
  uint64_t *k0 = nullptr, *k1 = nullptr;
  cudaError_t e = alloc_keys(nk, &k0, &k1);
  if (e != cudaSuccess) return e;
  k_rmat_keys<<<grid_for(samples), TPB, 0, st>>>(samples, scale, seed, tA, tAB, tABC, k0);
  if ((e = cudaGetLastError()) != cudaSuccess) {
    cudaFree(k0);
    cudaFree(k1);
    return e;
  }
  return build_from_keys(k0, k1, nk, int64_t(1) << scale, scale, seed, weighted, w_lo, w_hi, off64, st, out);
}

cudaError_t gen_sbm_device(int64_t n, int64_t k, int64_t samples, uint32_t fin24, uint64_t seed, bool off64,
                           cudaStream_t st, GenDeviceOut *out) {
  *out = GenDeviceOut{};
  int bits = 1;
  while ((int64_t(1) << bits) < n) ++bits;
  const int64_t nk = 2 * samples;
  uint64_t *k0 = nullptr, *k1 = nullptr;
  cudaError_t e = alloc_keys(nk, &k0, &k1);
  if (e != cudaSuccess) return e;
  k_sbm_keys<<<grid_for(samples), TPB, 0, st>>>(samples, n, k, fin24, seed, bits, k0);
  if ((e = cudaGetLastError()) != cudaSuccess) {
    cudaFree(k0);
    cudaFree(k1);
    return e;
  }
  return build_from_keys(k0, k1, nk, n, bits, seed, false, 1.0f, 1.0f, off64, st, out);
}

}  // namespace rak
