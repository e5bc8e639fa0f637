// rak_noalloc.cu -- rak_lowmem_cuda_noalloc: a complete νMG-/νBM-LPA run on a device-resident graph
// that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a process whose device memory has been handed almost
// entirely to a framework's pooling allocator (cudaMalloc then fails), or a caller on a
// latency-critical loop where cudaMalloc/cudaFree would add device-wide synchronisation. For them
// every working buffer of the run -- affected flags, the degree-bucket plan and its sort space,
// the split-vertex tables, partial sketches and arrival counters, per-iteration counters -- is
// carved out of one file-scope device array of RAK_NOALLOC_SCRATCH_BYTES. Graphs whose buffers do
// not fit are refused. The caller still passes the graph, the optional initial labels and flags,
// and the membership output, all on the device.
//
// The array is shared by every call in the process on a given device and keeps whatever the last
// call left in it: each call clears what must start at zero, and calls that overlap on the GPU
// (other streams, other host threads) race on it. The array's device address is looked up once
// per device, by the first call on that device, with that device current; make that first call
// before any stream capture. CUDA loads code and places __device__ arrays lazily: this file's
// module (and with it the array) is put on a device by that first call, and each kernel variant
// the call launches (slot count, mode, offset width, weighted or unit) by the first call that uses
// it. Those loads are the runtime's own device allocations, so a caller that is about to hand the
// device's memory to a pool makes one call of each variant it will use first. The caller's current
// device is restored before returning.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>

#include "rak_internal.hpp"
#include "rak_lowmem.h"

namespace rak {
namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[RAK_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 128;
std::mutex g_noalloc_mu;
void *g_noalloc_addr[kMaxDevices];

// Device address of the scratch array on `device` (current), looked up on first use.
rak_status scratch_base(int device, unsigned char **out) {
  if (device < 0 || device >= kMaxDevices) return RAK_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return RAK_ERR_CUDA;
    g_noalloc_addr[device] = p;
  }
  *out = static_cast<unsigned char *>(g_noalloc_addr[device]);
  return RAK_OK;
}

// Bump allocation inside the scratch array; `need` keeps counting past the end so a refusal can
// report how many bytes the graph would take.
struct Carve {
  unsigned char *base;
  size_t used = 0, need = 0;
  template <class T> T *take(size_t count) {
    const size_t b = (count * sizeof(T) + 255) & ~size_t(255);
    T *p = used + b <= RAK_NOALLOC_SCRATCH_BYTES ? reinterpret_cast<T *>(base + used) : nullptr;
    used += b;
    if (used > need) need = used;
    return p;
  }
};

template <class O>
__global__ void k_hub_chunk_counts(const O *off, const uint32_t *order, int64_t nhub, int64_t chunk, int64_t *cnt) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t h = tid; h < nhub; h += nt) {
    const uint32_t u = order[h];
    const int64_t deg = int64_t(off[u + 1]) - int64_t(off[u]);
    cnt[h + 1] = (deg + chunk - 1) / chunk;
  }
  if (tid == 0) cnt[0] = 0;
}

__global__ void k_chunk_owner(const int64_t *first, int64_t nhub, uint32_t *chunk_hub) {
  const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, nt = int64_t(gridDim.x) * blockDim.x;
  for (int64_t h = tid; h < nhub; h += nt)
    for (int64_t c = first[h]; c < first[h + 1]; ++c) chunk_hub[c] = uint32_t(h);
}

inline int blocks_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  return int(b < 1 ? 1 : (b > 148 * 32 ? 148 * 32 : b));
}

// Restores the calling thread's current device on every return path.
struct DeviceGuard {
  int saved = -1;
  DeviceGuard() { if (cudaGetDevice(&saved) != cudaSuccess) { saved = -1; cudaGetLastError(); } }
  ~DeviceGuard() { if (saved >= 0) cudaSetDevice(saved); }
};

#define NA_TRY(expr)                                                      \
  do {                                                                    \
    const cudaError_t _e = (expr);                                        \
    if (_e != cudaSuccess) {                                              \
      return _e == cudaErrorMemoryAllocation ? RAK_ERR_OUT_OF_MEMORY : RAK_ERR_CUDA; \
    }                                                                     \
  } while (0)

}  // namespace
}  // namespace rak

extern "C" rak_status rak_lowmem_cuda_noalloc(int device, void *stream, const rak_csr *g, const uint32_t *q,
                                              const rak_options *o, uint32_t *membership, rak_result *res) {
  using namespace rak;
  if (!g || !membership || g->location != RAK_DEVICE) return RAK_ERR_INVALID_ARGUMENT;
  if (g->n < 0 || g->n >= (int64_t(1) << 31) || g->m < 0 || (g->offset_bits != 32 && g->offset_bits != 64) ||
      !g->offsets || (g->m > 0 && !g->targets) ||
      (g->offset_bits == 32 && g->m > int64_t(std::numeric_limits<int32_t>::max())))
    return RAK_ERR_INVALID_ARGUMENT;
  rak_options d;
  rak_options_default(&d);
  if (!o) o = &d;
  const int slots = o->slots;
  if (!(slots == 1 || slots == 2 || slots == 4 || slots == 8 || slots == 16)) return RAK_ERR_INVALID_ARGUMENT;
  const int mode = o->mode;
  if (mode < RAK_MODE_ASYNC || mode > RAK_MODE_SYNC_SPLIT) return RAK_ERR_INVALID_ARGUMENT;
  const bool exact = mode == RAK_MODE_SYNC, sync = mode != RAK_MODE_ASYNC;
  const int rescan = o->rescan < 0 ? (exact ? 1 : 0) : (o->rescan ? 1 : 0);
  if (rescan && !exact && slots > 1) return RAK_ERR_UNSUPPORTED;
  if (o->sketch_rule > 2 || o->label_order > 2) return RAK_ERR_INVALID_ARGUMENT;
  if (exact && o->sketch_rule == 2) return RAK_ERR_UNSUPPORTED;
  // labels as in rak_lowmem_cuda: vertex ids by default (the reference GPU path's vertex order for
  // asynchronous runs with one or two slots); label_order 2 (asynchronous runs) takes positions in that
  // order, two n-sized tables more in the array
  const int order_kind = o->label_order <= 0 ? default_label_order(mode, slots) : o->label_order;
  if (order_kind == 2 && sync) return RAK_ERR_UNSUPPORTED;
  const int iters = o->max_iterations;
  if (iters < 0 || iters > 1024 || !(o->tolerance >= 0) || o->wait_timeout_ns < 0) return RAK_ERR_INVALID_ARGUMENT;
  if (o->tie_break > 2 || o->tie_iterations < 0 || o->edge_staging > 2 || o->dense_pct > 100) return RAK_ERR_INVALID_ARGUMENT;
  if (o->tie_break == 2 && o->sketch_rule == 2) return RAK_ERR_UNSUPPORTED;
  Layout ly;
  ly.lane_max = o->lane_max > 0 ? o->lane_max : DEFAULT_LANE_MAX;
  ly.hub_min = o->hub_min > 0 ? o->hub_min : DEFAULT_HUB_MIN;
  ly.hub_chunk = o->hub_chunk > 0 ? o->hub_chunk : DEFAULT_HUB_CHUNK;
  if (ly.lane_max > MAX_LANE_MAX || ly.hub_min < ly.lane_max || ly.hub_chunk < 32) return RAK_ERR_INVALID_ARGUMENT;
  rak_result tmp;
  rak_result *rr = res ? res : &tmp;
  std::memset(rr, 0, sizeof(*rr));
  rr->modularity = std::numeric_limits<double>::quiet_NaN();

  DeviceGuard keep_device;
  NA_TRY(cudaSetDevice(device));
  unsigned char *base = nullptr;
  rak_status s = scratch_base(device, &base);
  if (s != RAK_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = g->n;
  const bool off64 = g->offset_bits == 64;
  const auto t0 = std::chrono::steady_clock::now();

  Carve cv{base};
  unsigned int *bad = cv.take<unsigned int>(1);
  uint32_t *order = cv.take<uint32_t>(size_t(n > 0 ? n : 1));
  const bool ref_labels = order_kind == 2 && n > 0;
  uint32_t *ref_ks = ref_labels ? cv.take<uint32_t>(size_t(n)) : nullptr;
  uint32_t *ref_pos = ref_labels ? cv.take<uint32_t>(size_t(n)) : nullptr;
  const size_t plan_mark = cv.used;

  // ---- plan: per-vertex keys, stable radix sort into regions, key histogram -------------------
  const int nk = int(6 + ly.lane_max + 1);
  uint32_t *keys = cv.take<uint32_t>(size_t(n > 0 ? n : 1));
  uint32_t *keys2 = cv.take<uint32_t>(size_t(n > 0 ? n : 1));
  uint32_t *vids = cv.take<uint32_t>(size_t(n > 0 ? n : 1));
  unsigned long long *hist = cv.take<unsigned long long>(size_t(nk));
  int end_bit = 1;
  while ((1 << end_bit) < nk) ++end_bit;
  size_t sort_bytes = 0;
  if (n > 0) NA_TRY(plan_sort(nullptr, nullptr, nullptr, nullptr, n, end_bit, nullptr, &sort_bytes, st));
  void *sort_tmp = cv.take<unsigned char>(sort_bytes > 0 ? sort_bytes : 1);
  if (cv.need > RAK_NOALLOC_SCRATCH_BYTES) { rr->peak_device_bytes = cv.need; return RAK_ERR_OUT_OF_MEMORY; }
  if (o->validate) {
    unsigned int hbad = 0;
    NA_TRY(cudaMemsetAsync(bad, 0, sizeof(unsigned int), st));
    NA_TRY(launch_validate(g->offsets, off64, g->targets, n, g->m, bad, st));
    NA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, st));
    NA_TRY(cudaStreamSynchronize(st));
    if (hbad) return RAK_ERR_INVALID_CSR;
  }
  unsigned long long h[6 + MAX_LANE_MAX + 1];
  std::memset(h, 0, sizeof(h));
  NA_TRY(cudaMemsetAsync(hist, 0, size_t(nk) * sizeof(unsigned long long), st));
  if (n > 0) {
    NA_TRY(launch_plan_keys(g->offsets, off64, n, ly, keys, vids, hist, nk, st));
    NA_TRY(plan_sort(keys, keys2, vids, order, n, end_bit, sort_tmp, &sort_bytes, st));
    NA_TRY(cudaMemcpyAsync(h, hist, size_t(nk) * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    NA_TRY(cudaStreamSynchronize(st));
  }
  cv.used = plan_mark;  // sort space is dead from here on
  if (ref_labels) {
    // the reference order (depends on degrees only), built in the dead sort space
    void *ref_tmp = cv.take<unsigned char>(ref_order_scratch_bytes(n, 1));
    if (cv.need > RAK_NOALLOC_SCRATCH_BYTES) { rr->peak_device_bytes = cv.need; return RAK_ERR_OUT_OF_MEMORY; }
    NA_TRY(ref_order(g->offsets, off64, n, nullptr, nullptr, 0, ref_ks, ref_pos, ref_tmp, st));
    NA_TRY(cudaStreamSynchronize(st));
    cv.used = plan_mark;
  }

  // ---- split-vertex chunk tables, built on the device --------------------------------------------
  const int64_t nhub = int64_t(h[0]);
  int64_t nchunks = 0;
  int64_t *first = cv.take<int64_t>(size_t(nhub + 1));
  if (!first) { rr->peak_device_bytes = cv.need; return RAK_ERR_OUT_OF_MEMORY; }
  if (nhub > 0) {
    const size_t mark = cv.used;
    int64_t *cnt = cv.take<int64_t>(size_t(nhub + 1));
    size_t scan_bytes = 0;
    NA_TRY(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, cnt, first, nhub + 1, st));
    void *scan_tmp = cv.take<unsigned char>(scan_bytes > 0 ? scan_bytes : 1);
    if (!cnt || !scan_tmp) { rr->peak_device_bytes = cv.need; return RAK_ERR_OUT_OF_MEMORY; }
    if (off64) k_hub_chunk_counts<int64_t><<<blocks_for(nhub), 256, 0, st>>>(static_cast<const int64_t *>(g->offsets), order, nhub, ly.hub_chunk, cnt);
    else k_hub_chunk_counts<int32_t><<<blocks_for(nhub), 256, 0, st>>>(static_cast<const int32_t *>(g->offsets), order, nhub, ly.hub_chunk, cnt);
    NA_TRY(cudaGetLastError());
    NA_TRY(cub::DeviceScan::InclusiveSum(scan_tmp, scan_bytes, cnt, first, nhub + 1, st));
    NA_TRY(cudaMemcpyAsync(&nchunks, first + nhub, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    NA_TRY(cudaStreamSynchronize(st));
    cv.used = mark;
  }
  uint32_t *chunk_hub = cv.take<uint32_t>(size_t(nchunks > 0 ? nchunks : 1));
  Regions rg{};
  {
    int64_t cnt[NREG] = {};
    for (int k = 0; k < 6; ++k) cnt[k] = int64_t(h[k]);
    for (int64_t k = 6; k < 6 + ly.lane_max; ++k) cnt[REG_LANE] += int64_t(h[k]);
    int sms = 0;
    NA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    rg.lane_item = lane_item_for(cnt[REG_LANE], int64_t(sms) * LPA_WARPS_PER_SM);
    int64_t v = 0, it = 0;
    for (int r = 0; r < NREG; ++r) {
      rg.vbegin[r] = v;
      rg.vcount[r] = cnt[r];
      v += cnt[r];
      rg.ibegin[r] = it;
      it += region_items(r, cnt[r], nchunks, rg.lane_item);
    }
    rg.ibegin[NREG] = it;
  }

  // ---- run buffers ---------------------------------------------------------------------------------
  const int it_slots = iters > 0 ? iters : 1;
  uint8_t *aff0 = cv.take<uint8_t>(size_t(n) + 16);
  uint8_t *aff1 = sync ? cv.take<uint8_t>(size_t(n) + 16) : nullptr;
  uint32_t *vcom1 = sync ? cv.take<uint32_t>(size_t(n) + 4) : nullptr;
  uint32_t *arrive = cv.take<uint32_t>(size_t(nhub > 0 ? nhub : 1));
  uint32_t *claim = cv.take<uint32_t>(size_t(nhub > 0 ? nhub : 1));
  int32_t *moved = cv.take<int32_t>(size_t(nhub > 0 ? nhub : 1));
  uint32_t *skk = cv.take<uint32_t>(size_t(nchunks > 0 ? nchunks : 1) * size_t(slots));
  float *skw = cv.take<float>(size_t(nchunks > 0 ? nchunks : 1) * size_t(slots));
  unsigned long long *stats = cv.take<unsigned long long>(size_t(it_slots) * STATS_STRIDE);
  RunStateHost *rs = cv.take<RunStateHost>(1);
  if (cv.need > RAK_NOALLOC_SCRATCH_BYTES) { rr->peak_device_bytes = cv.need; return RAK_ERR_OUT_OF_MEMORY; }
  if (nhub > 0) {
    k_chunk_owner<<<blocks_for(nhub), 256, 0, st>>>(first, nhub, chunk_hub);
    NA_TRY(cudaGetLastError());
  }
  NA_TRY(cudaMemsetAsync(arrive, 0, size_t(nhub > 0 ? nhub : 1) * 4, st));
  NA_TRY(cudaMemsetAsync(claim, 0, size_t(nhub > 0 ? nhub : 1) * 4, st));
  NA_TRY(cudaMemsetAsync(moved, 0xFF, size_t(nhub > 0 ? nhub : 1) * 4, st));
  NA_TRY(cudaMemsetAsync(stats, 0, size_t(it_slots) * STATS_STRIDE * 8, st));
  NA_TRY(cudaMemsetAsync(rs, 0, sizeof(RunStateHost), st));
  // the kernel's code is loaded (CUDA loads modules lazily) before the timed part
  const bool stage = (o->edge_staging <= 0 ? DEFAULT_EDGE_STAGING : o->edge_staging) == 1;
  if (iters > 0) NA_TRY(prepare_lpa(slots, mode, off64, g->weights == nullptr, false, stage));
  const auto t1 = std::chrono::steady_clock::now();
  if (ref_labels) NA_TRY(launch_init_mapped(membership, q, ref_pos, n, st));
  else NA_TRY(launch_init(membership, vcom1, q, n, st));
  NA_TRY(launch_init_flags(aff0, aff1, o->initial_flags, n, st));
  LpaArgs a{};
  a.off = g->offsets; a.tgt = g->targets; a.wt = g->weights; a.n = n;
  a.order = order; a.rg = rg;
  a.chunk_hub = chunk_hub; a.hub_first = first; a.hub_chunk = ly.hub_chunk; a.nchunks = nchunks;
  a.vcom0 = membership; a.vcom1 = vcom1; a.aff0 = aff0; a.aff1 = aff1;
  a.hub_arrive = arrive; a.hub_claim = claim; a.hub_moved = moved; a.sk_keys = skk; a.sk_wts = skw;
  a.stats = stats; a.rs = rs;
  a.iters = iters; a.start_iter = o->start_iteration; a.tolerance = o->tolerance;
  a.pickless_step = o->pickless_step < 0 ? (mode == RAK_MODE_ASYNC ? 8 : 0) : o->pickless_step;
  a.check_on_pickless = o->check_on_pickless < 0 ? (mode == RAK_MODE_ASYNC ? 0 : 1) : (o->check_on_pickless ? 1 : 0);
  a.rescan = rescan;
  a.mark_test = mark_test_for(n, g->m);
  // rule sets as in rak_lowmem_cuda: the CPU rules unless sketch_rule asks for the GPU ones
  a.gpu_rule = mode != RAK_MODE_SYNC && o->sketch_rule == 2;
  // ties as in rak_lowmem_cuda: hashed during the first iterations of asynchronous runs
  const int tie = o->tie_break <= 0 ? (mode == RAK_MODE_ASYNC && !a.gpu_rule ? 2 : 1) : o->tie_break;
  a.tie_until = tie == 2 ? (o->tie_iterations > 0 ? o->tie_iterations : DEFAULT_TIE_ITERATIONS) : 0;
  a.stage = stage;
  a.grid_cap = o->max_blocks > 0 ? o->max_blocks : 0;
  a.timeout_ns = o->wait_timeout_ns > 0 ? (long long)o->wait_timeout_ns : DEFAULT_WAIT_TIMEOUT_NS;
  a.dense_moved_edges = dense_threshold(mode, o->dense_pct, g->m);
  if (iters > 0) {
    int grid = 0;
    NA_TRY(launch_lpa(a, slots, mode, off64, st, &grid));
  }
  RunStateHost hs{};
  unsigned long long sh[1024 * STATS_STRIDE];
  NA_TRY(cudaMemcpyAsync(&hs, rs, sizeof(hs), cudaMemcpyDeviceToHost, st));
  NA_TRY(cudaMemcpyAsync(sh, stats, size_t(it_slots) * STATS_STRIDE * 8, cudaMemcpyDeviceToHost, st));
  NA_TRY(cudaStreamSynchronize(st));
  if (hs.error) return rak_status(hs.error);
  const int done = iters > 0 ? int(hs.iterations) : 0;
  if (sync && (done & 1)) {
    NA_TRY(cudaMemcpyAsync(membership, vcom1, size_t(n) * 4, cudaMemcpyDeviceToDevice, st));
    NA_TRY(cudaStreamSynchronize(st));
  }
  if (ref_labels) {
    NA_TRY(launch_labels_to_ids(membership, ref_ks, n, st));
    NA_TRY(cudaStreamSynchronize(st));
  }
  const auto t2 = std::chrono::steady_clock::now();
  rr->iterations = done;
  rr->time_ms = float(std::chrono::duration<double, std::milli>(t2 - t1).count());
  rr->loop_ms = rr->time_ms;
  rr->plan_ms = float(std::chrono::duration<double, std::milli>(t1 - t0).count());
  for (int i = 0; i < done; ++i) {
    const unsigned long long *x = sh + size_t(i) * STATS_STRIDE;
    rr->traversed_edges += x[STAT_EDGES];
    rr->processed_vertices += x[STAT_PROCESSED];
    rr->moved_vertices += x[STAT_CHANGED];
    rr->moved_edges += x[STAT_MOVED_EDGES];
    if (x[STAT_PHASE] & 1ull) rr->dense_iterations += 1;
    else rr->marked_edges += x[STAT_MOVED_EDGES];
  }
  rr->changed_last = done > 0 ? sh[size_t(done - 1) * STATS_STRIDE + STAT_CHANGED] : 0;
  rr->peak_device_bytes = cv.need;
  rr->memory_gb = float(double(cv.need) / (1024.0 * 1024.0 * 1024.0));
  if (o->compute_modularity && n > 0) {
    cv.used = plan_mark;  // run buffers are dead: reuse them
    double *ctot = cv.take<double>(size_t(n));
    double *sums = cv.take<double>(4);
    if (!ctot || !sums) { rr->peak_device_bytes = cv.need; return RAK_ERR_OUT_OF_MEMORY; }
    double hm[4] = {0, 0, 0, 0};
    NA_TRY(cudaMemsetAsync(ctot, 0, size_t(n) * 8, st));
    NA_TRY(cudaMemsetAsync(sums, 0, 4 * 8, st));
    NA_TRY(launch_modularity(g->offsets, off64, g->targets, g->weights, n, membership, ctot, sums, st));
    NA_TRY(cudaMemcpyAsync(hm, sums, sizeof(hm), cudaMemcpyDeviceToHost, st));
    NA_TRY(cudaStreamSynchronize(st));
    if (hm[3] > 0) return RAK_ERR_INVALID_ARGUMENT;  // labels >= n (from q) are not vertex ids
    rr->modularity = hm[1] > 0 ? hm[0] / hm[1] - hm[2] / (hm[1] * hm[1]) : 0.0;
    rr->peak_device_bytes = cv.need;
  }
  return RAK_OK;
}
