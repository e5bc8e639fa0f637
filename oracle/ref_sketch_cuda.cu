// ref_sketch_cuda.cu -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own GPU Misra-Gries sketch functions (inc/sketchCuda.hxx:
// sketchAccumulateWarpCudU :73-108, the accumulate its group kernel uses for SLOTS <= 32,
// inc/rakLowmemCuda.hxx:272, 82-83; sketchMaxGroupReduceCudU :190-201) on streams of
// (community, weight) pairs, so the oracle's restatement of those rules can be checked against the
// reference's code itself. Each stream starts from cleared keys (NONE) and zero weights, one
// SLOTS-thread tile per stream, one call per pair in stream order, as the reference's scan loop
// makes them (inc/rakLowmemCuda.hxx:75-87). With slots 1 it runs the reference's Boyer-Moore scan,
// rakLowmemBmScanCommunitiesCud (inc/rakLowmemCuda.hxx:38-54), from the given own label of each
// stream's vertex, over a CSR built so that stream i is vertex i's edge list (targets offset past
// the stream indices, so no edge is a self-loop). Built by oracle/Makefile into oracle/_ref from
// the reference headers in place; a separate process, like ref_lpa_cuda.
//
// usage: ref_sketch_cuda <streams.in> <sketches.out>
// in:  "RAKSKT01", int32 slots (1, 2, 4, 8 or 16), int64 streams, int64 total,
//      int64 offsets[streams+1], uint32 communities[total], float weights[total],
//      and for slots 1: uint32 own_label[streams]
// out: uint32 keys[streams*slots], float weights[streams*slots] (the sketch before the argmax),
//      uint32 best_key[streams], float best_weight[streams] (slot 0 after the tournament; for
//      slots 1 the Boyer-Moore candidate and its weight in both places)
#define BUILD 0
#define OPENMP 0
#define CUDA 1
#include <cooperative_groups.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "_main.hxx"
#include "csr.hxx"
#include "properties.hxx"
#include "sketchCuda.hxx"
#include "rak.hxx"
#include "rakCuda.hxx"
#include "rakLowmemCuda.hxx"

namespace {

template <int S>
__global__ void k_streams(const int64_t *off, const uint32_t *comm, const float *wts, int64_t ns, uint32_t *okeys,
                          float *owts, uint32_t *bestk, float *bestw) {
  const auto g = cooperative_groups::tiled_partition<S>(cooperative_groups::this_thread_block());
  const int s = int(threadIdx.x);  // blockDim.x == S: one tile per block
  __shared__ uint32_t mcs[S];
  __shared__ float mws[S];
  for (int64_t i = blockIdx.x; i < ns; i += gridDim.x) {
    mcs[s] = 0xFFFFFFFFu;
    mws[s] = 0.0f;
    g.sync();
    for (int64_t e = off[i]; e < off[i + 1]; ++e) sketchAccumulateWarpCudU<false>(mcs, mws, comm[e], wts[e], g, s);
    g.sync();
    okeys[i * S + s] = mcs[s];
    owts[i * S + s] = mws[s];
    g.sync();
    sketchMaxGroupReduceCudU(mcs, mws, S, g, s);
    g.sync();
    if (s == 0) {
      bestk[i] = mcs[0];
      bestw[i] = mws[0];
    }
    g.sync();
  }
}

// One thread per stream: vertex i's edges are xedg[off[i]..off[i+1]), with labels vcom[xedg[e]].
__global__ void k_bm(const int64_t *off, const uint32_t *xedg, const float *wts, const uint32_t *vcom,
                     const uint32_t *own, int64_t ns, uint32_t *bestk, float *bestw) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < ns; i += int64_t(gridDim.x) * blockDim.x) {
    auto mcw = rakLowmemBmScanCommunitiesCud<false>(off, xedg, wts, vcom, uint32_t(i), own[i], int64_t(0), int64_t(1));
    bestk[i] = mcw.first;
    bestw[i] = mcw.second;
  }
}

bool check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
  return false;
}

template <class T>
bool read_n(FILE *f, T *p, size_t n) {
  return n == 0 || std::fread(p, sizeof(T), n, f) == n;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: ref_sketch_cuda <streams.in> <sketches.out>\n");
    return 2;
  }
  FILE *f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  char magic[8];
  int32_t slots = 0;
  int64_t ns = 0, total = 0;
  if (!read_n(f, magic, 8) || std::memcmp(magic, "RAKSKT01", 8) != 0 || !read_n(f, &slots, 1) ||
      !read_n(f, &ns, 1) || !read_n(f, &total, 1) || ns < 0 || total < 0 ||
      !(slots == 1 || slots == 2 || slots == 4 || slots == 8 || slots == 16)) {
    std::fclose(f);
    return 2;
  }
  std::vector<int64_t> off(static_cast<size_t>(ns) + 1);
  std::vector<uint32_t> comm(static_cast<size_t>(total));
  std::vector<float> wts(static_cast<size_t>(total));
  std::vector<uint32_t> own(slots == 1 ? static_cast<size_t>(ns) : 0);
  const bool ok = read_n(f, off.data(), off.size()) && read_n(f, comm.data(), comm.size()) &&
                  read_n(f, wts.data(), wts.size()) && read_n(f, own.data(), own.size());
  std::fclose(f);
  if (!ok || off[0] != 0 || off[size_t(ns)] != total) return 2;
  for (int64_t i = 0; i < ns; ++i)
    if (off[size_t(i) + 1] < off[size_t(i)]) return 2;
  const size_t nk = size_t(ns) * size_t(slots);
  std::vector<uint32_t> okeys(nk), bestk(static_cast<size_t>(ns));
  std::vector<float> owts(nk), bestw(static_cast<size_t>(ns));
  if (ns > 0) {
    int64_t *d_off = nullptr;
    uint32_t *d_comm = nullptr, *d_okeys = nullptr, *d_bestk = nullptr;
    float *d_wts = nullptr, *d_owts = nullptr, *d_bestw = nullptr;
    const size_t te = size_t(total > 0 ? total : 1);
    if (!check(cudaMalloc(&d_off, off.size() * 8), "cudaMalloc") || !check(cudaMalloc(&d_comm, te * 4), "cudaMalloc") ||
        !check(cudaMalloc(&d_wts, te * 4), "cudaMalloc") || !check(cudaMalloc(&d_okeys, nk * 4), "cudaMalloc") ||
        !check(cudaMalloc(&d_owts, nk * 4), "cudaMalloc") || !check(cudaMalloc(&d_bestk, size_t(ns) * 4), "cudaMalloc") ||
        !check(cudaMalloc(&d_bestw, size_t(ns) * 4), "cudaMalloc"))
      return 1;
    if (!check(cudaMemcpy(d_off, off.data(), off.size() * 8, cudaMemcpyHostToDevice), "copy") ||
        (total > 0 && !check(cudaMemcpy(d_comm, comm.data(), size_t(total) * 4, cudaMemcpyHostToDevice), "copy")) ||
        (total > 0 && !check(cudaMemcpy(d_wts, wts.data(), size_t(total) * 4, cudaMemcpyHostToDevice), "copy")))
      return 1;
    const unsigned grid = unsigned(ns < 4096 ? ns : 4096);
    if (slots == 1) {
      // stream i is vertex i; edge e targets vertex ns + e, whose label is communities[e]
      std::vector<uint32_t> xedg(te), vcom(size_t(ns) + te, 0u);
      for (int64_t e = 0; e < total; ++e) {
        xedg[size_t(e)] = uint32_t(ns + e);
        vcom[size_t(ns + e)] = comm[size_t(e)];
      }
      uint32_t *d_xedg = nullptr, *d_vcom = nullptr, *d_own = nullptr;
      if (!check(cudaMalloc(&d_xedg, te * 4), "cudaMalloc") ||
          !check(cudaMalloc(&d_vcom, (size_t(ns) + te) * 4), "cudaMalloc") ||
          !check(cudaMalloc(&d_own, size_t(ns) * 4), "cudaMalloc") ||
          !check(cudaMemcpy(d_xedg, xedg.data(), te * 4, cudaMemcpyHostToDevice), "copy") ||
          !check(cudaMemcpy(d_vcom, vcom.data(), (size_t(ns) + te) * 4, cudaMemcpyHostToDevice), "copy") ||
          !check(cudaMemcpy(d_own, own.data(), size_t(ns) * 4, cudaMemcpyHostToDevice), "copy"))
        return 1;
      k_bm<<<(unsigned(ns) + 127) / 128 < 4096 ? (unsigned(ns) + 127) / 128 : 4096, 128>>>(
          d_off, d_xedg, d_wts, d_vcom, d_own, ns, d_bestk, d_bestw);
      if (!check(cudaGetLastError(), "launch") || !check(cudaDeviceSynchronize(), "run")) return 1;
      if (!check(cudaMemcpy(d_okeys, d_bestk, size_t(ns) * 4, cudaMemcpyDeviceToDevice), "copy") ||
          !check(cudaMemcpy(d_owts, d_bestw, size_t(ns) * 4, cudaMemcpyDeviceToDevice), "copy"))
        return 1;
      cudaFree(d_xedg); cudaFree(d_vcom); cudaFree(d_own);
    }
    switch (slots) {
      case 1: break;
      case 2: k_streams<2><<<grid, 2>>>(d_off, d_comm, d_wts, ns, d_okeys, d_owts, d_bestk, d_bestw); break;
      case 4: k_streams<4><<<grid, 4>>>(d_off, d_comm, d_wts, ns, d_okeys, d_owts, d_bestk, d_bestw); break;
      case 8: k_streams<8><<<grid, 8>>>(d_off, d_comm, d_wts, ns, d_okeys, d_owts, d_bestk, d_bestw); break;
      default: k_streams<16><<<grid, 16>>>(d_off, d_comm, d_wts, ns, d_okeys, d_owts, d_bestk, d_bestw); break;
    }
    if (!check(cudaGetLastError(), "launch") || !check(cudaDeviceSynchronize(), "run")) return 1;
    if (!check(cudaMemcpy(okeys.data(), d_okeys, nk * 4, cudaMemcpyDeviceToHost), "copy") ||
        !check(cudaMemcpy(owts.data(), d_owts, nk * 4, cudaMemcpyDeviceToHost), "copy") ||
        !check(cudaMemcpy(bestk.data(), d_bestk, size_t(ns) * 4, cudaMemcpyDeviceToHost), "copy") ||
        !check(cudaMemcpy(bestw.data(), d_bestw, size_t(ns) * 4, cudaMemcpyDeviceToHost), "copy"))
      return 1;
    cudaFree(d_off); cudaFree(d_comm); cudaFree(d_wts); cudaFree(d_okeys); cudaFree(d_owts);
    cudaFree(d_bestk); cudaFree(d_bestw);
  }
  FILE *o = std::fopen(argv[2], "wb");
  if (!o) return 2;
  std::fwrite(okeys.data(), 4, nk, o);
  std::fwrite(owts.data(), 4, nk, o);
  std::fwrite(bestk.data(), 4, size_t(ns), o);
  std::fwrite(bestw.data(), 4, size_t(ns), o);
  std::fclose(o);
  return 0;
}
