// rak_host.cpp -- host orchestration behind the C ABI (include/rak_lowmem.h): contexts, device
// residency of graphs, the degree-bucket plan, runs, single steps and modularity.
//
// Reference path replaced: rakLowmemInvokeCuda (inc/rakLowmemCuda.hxx:538-607) and
// rakLowmemStaticCuda (:624-632). The reference partitions vertices on the host into
// degree < 4 | < 128 | >= 128 (rakLowmemPartitionVerticesCudaU, :505-519), builds a permuted CSR
// on the host and copies it; here the graph is copied as given and the bucketing is a device-side
// radix sort of per-vertex keys (no CSR rewrite), producing the work regions of rak_internal.hpp.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "rak_internal.hpp"
#include "rak_lowmem.h"

struct rak_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own = nullptr;
  int sms = 0;
  std::string err;
  cudaMemPool_t pool = nullptr;  // one-shot runs allocate here while keep > 0 (rak_ctx_set_memory_keep)
  uint64_t keep = 0;
};

namespace rak_host_detail {

// Device allocation that frees itself, with byte accounting for peak_device_bytes.
struct Tracker {
  uint64_t cur = 0, peak = 0;
  void add(uint64_t b) { cur += b; peak = std::max(peak, cur); }
  void sub(uint64_t b) { cur -= std::min(cur, b); }
};

// Where this thread's device allocations come from: cudaMalloc (no pool), or stream-ordered from
// a memory pool on a stream (PoolScope). The server's launch slots use their own pools, so that
// growing a slot's buffers never waits for the whole device (cudaFree does).
struct PoolTarget {
  cudaMemPool_t pool = nullptr;
  cudaStream_t stream = nullptr;
};
inline PoolTarget &thread_pool() {
  static thread_local PoolTarget t;
  return t;
}
struct PoolScope {
  PoolTarget saved;
  PoolScope(cudaMemPool_t pool, cudaStream_t stream) : saved(thread_pool()) { thread_pool() = {pool, stream}; }
  ~PoolScope() { thread_pool() = saved; }
};

// Allocates from the current PoolScope's pool, else with cudaMalloc.
inline cudaError_t dev_alloc(void **p, size_t bytes, cudaStream_t *freed_on) {
  const PoolTarget &pt = thread_pool();
  *freed_on = pt.stream;
  if (pt.pool) return cudaMallocFromPoolAsync(p, bytes, pt.pool, pt.stream);
  return cudaMalloc(p, bytes);
}
inline void dev_free(void *p, bool pooled, cudaStream_t freed_on) {
  if (!p) return;
  if (pooled) cudaFreeAsync(p, freed_on);
  else cudaFree(p);
}

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  Tracker *t = nullptr;
  bool pooled = false;
  cudaStream_t fs = nullptr;  // stream a pooled buffer is freed on
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) { dev_free(p, pooled, fs); if (t) t->sub(bytes); }
    p = nullptr;
    bytes = 0;
    pooled = false;
  }
  cudaError_t alloc(size_t b, Tracker *tr) {
    release();
    bytes = b ? b : 16;
    t = tr;
    pooled = thread_pool().pool != nullptr;
    cudaError_t e = dev_alloc(&p, bytes, &fs);
    if (e != cudaSuccess) { p = nullptr; bytes = 0; pooled = false; return e; }
    if (t) t->add(bytes);
    return e;
  }
  template <class T> T *as() const { return static_cast<T *>(p); }
};

// Per-run device buffers, kept by a resident graph and reused while large enough.
struct RunBufs {
  DevBuf vcom1, aff0, aff1, arrive, claim, moved, skk, skw, stats, rs;
  DevBuf lab;   // labels of a renumbered run, in the renumbered graph's numbering
  uint64_t bytes() const {
    return vcom1.bytes + aff0.bytes + aff1.bytes + arrive.bytes + claim.bytes + moved.bytes + skk.bytes +
           skw.bytes + stats.bytes + rs.bytes + lab.bytes;
  }
};

}  // namespace rak_host_detail

struct rak_graph {
  rak_ctx *ctx = nullptr;
  int device = 0;                   // kept here: the context may be destroyed first
  int64_t n = 0, m = 0;
  bool off64 = false;
  bool owns = false;  // graph arrays copied by us (freed on destroy)
  const void *off = nullptr;
  const uint32_t *tgt = nullptr;
  const float *wt = nullptr;
  rak::Layout ly{0, 0, 0};
  uint32_t *order = nullptr;
  uint32_t *chunk_hub = nullptr;
  int64_t *hub_first = nullptr;
  int64_t nhub = 0, nchunks = 0;
  rak::Regions rg{};
  uint64_t graph_bytes = 0, plan_bytes = 0;  // allocated by the library: graph copy, plan
  uint64_t ref_bytes = 0;                    // the caller's device arrays a device-located graph uses
  float plan_ms = 0, h2d_ms = 0;
  size_t off_cap = 0, tgt_cap = 0, wt_cap = 0;  // bytes allocated for an owned copy
  void *wt_alloc = nullptr;                      // owned weight buffer (wt may be null: unit weights)
  bool arrays_pooled = false;                    // owned arrays come from a server slot's pool
  cudaStream_t arrays_fs = nullptr;              // ... and are freed on this stream
  rak_host_detail::RunBufs bufs;  // run buffers reused across runs
  // plan storage (order and split-vertex tables) and its build space, grown only when too small
  rak_host_detail::DevBuf p_order, p_hub_first, p_chunk_hub, p_keys, p_keys2, p_vids, p_hist, p_temp, p_deg;
  // the reference GPU path's vertex order (asynchronous runs name labels by position in it)
  rak_host_detail::DevBuf ref_ks, ref_pos;
  bool ref_ready = false;
  // the graph renumbered in the plan's work order (rak_options.renumber), built at the first run
  // that uses it: old -> new ids, offsets, targets, weights, and the identity work order
  rak_host_detail::DevBuf rn_inv, rn_off, rn_tgt, rn_wt, rn_ident;
  bool rn_ready = false;
  rak::Layout rn_ly{0, 0, 0};
  uint64_t rn_bytes() const { return rn_inv.bytes + rn_off.bytes + rn_tgt.bytes + rn_wt.bytes + rn_ident.bytes; }
};

struct rak_batch {
  rak_ctx *ctx = nullptr;
  int device = 0;
  rak_graph *g = nullptr;           // the concatenated CSR (64-bit offsets) and its plan
  int64_t ngraphs = 0;
  rak_host_detail::DevBuf vbase, gid, vcom0, gdone, giters, gchanged, running;
  rak_host_detail::DevBuf ref_ks, ref_pos;  // every graph's reference vertex order (global indices)
  rak_host_detail::DevBuf ref_scratch;      // the order's work space (kept only by server slots)
  bool ref_ready = false;
  bool keep_ref_scratch = false;            // server slots rebuild the order for every packed set
  int last_iters = 0;               // max_iterations of the last launch
  bool last_sync = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

using rak::Layout;
using rak_host_detail::DevBuf;
using rak_host_detail::RunBufs;
using rak_host_detail::Tracker;

// Reuses a cached buffer when it is large enough (untracked: it outlives the call).
// Grows d to at least `bytes` (contents are not kept). A buffer that has to grow again gets half
// as much again, so a series of slightly larger requests does not reallocate every time.
cudaError_t ensure(DevBuf &d, size_t bytes) {
  if (d.p && d.bytes >= bytes) return cudaSuccess;
  return d.alloc(d.p ? bytes + bytes / 2 : bytes, nullptr);
}

void set_err(rak_ctx *ctx, const char *fmt, ...) {
  if (!ctx) return;
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  ctx->err = buf;
}

rak_status from_cuda(rak_ctx *ctx, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return RAK_OK;
  set_err(ctx, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // not sticky: clear it
    return RAK_ERR_OUT_OF_MEMORY;
  }
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return RAK_ERR_NO_DEVICE;
  return RAK_ERR_CUDA;
}

#define RAK_TRY(ctx, expr)                                         \
  do {                                                             \
    rak_status _s = from_cuda((ctx), (expr), #expr);               \
    if (_s != RAK_OK) return _s;                                   \
  } while (0)
#define RAK_CHECK(expr)            \
  do {                             \
    rak_status _s = (expr);        \
    if (_s != RAK_OK) return _s;   \
  } while (0)

struct Events {
  cudaEvent_t e[6] = {};
  Events() { for (auto &x : e) cudaEventCreate(&x); }
  ~Events() { for (auto &x : e) if (x) cudaEventDestroy(x); }
  float ms(int a, int b) const {
    float t = 0;
    cudaEventElapsedTime(&t, e[a], e[b]);
    return t;
  }
};

struct Resolved {
  int slots, mode, rescan, pickless, check_on_pickless, iters, start, validate, modularity, repeat, rule, order;
  double tol;
  long long timeout_ns;  // bound on each device-side wait
  int tie_until;         // iterations with hashed Misra-Gries ties
  int stage;             // edge staging through shared memory
  int max_blocks;        // cap on the persistent launch's blocks (0: none)
  int dense_pct;         // rak_options.dense_pct as given (rak::dense_threshold resolves it)
  int renumber;          // runs on the graph renumbered in work order: 0 no, 1 large graphs, 2 yes
  bool one_shot = false; // rak_lowmem_cuda: the graph (and a renumbered copy) is built for one call
  Layout ly;
};

rak_status resolve(rak_ctx *ctx, const rak_options *o, Resolved *r) {
  rak_options d;
  rak_options_default(&d);
  if (!o) o = &d;
  r->slots = o->slots;
  if (!(r->slots == 1 || r->slots == 2 || r->slots == 4 || r->slots == 8 || r->slots == 16)) {
    set_err(ctx, "slots must be 1, 2, 4, 8 or 16 (got %d)", o->slots);
    return RAK_ERR_INVALID_ARGUMENT;
  }
  r->mode = o->mode;
  if (r->mode < RAK_MODE_ASYNC || r->mode > RAK_MODE_SYNC_SPLIT) { set_err(ctx, "bad mode %d", o->mode); return RAK_ERR_INVALID_ARGUMENT; }
  const bool sync = r->mode == RAK_MODE_SYNC;
  r->rescan = o->rescan < 0 ? (sync ? 1 : 0) : (o->rescan ? 1 : 0);
  if (r->rescan && !sync && r->slots > 1) {
    set_err(ctx, "rescan is implemented for RAK_MODE_SYNC only");
    return RAK_ERR_UNSUPPORTED;
  }
  r->pickless = o->pickless_step < 0 ? (r->mode == RAK_MODE_ASYNC ? 8 : 0) : o->pickless_step;
  r->check_on_pickless = o->check_on_pickless < 0 ? (r->mode == RAK_MODE_ASYNC ? 0 : 1) : (o->check_on_pickless ? 1 : 0);
  r->iters = o->max_iterations;
  if (r->iters < 0 || r->iters > 1024) { set_err(ctx, "max_iterations must be in [0, 1024]"); return RAK_ERR_INVALID_ARGUMENT; }
  r->tol = o->tolerance;
  if (!(r->tol >= 0)) { set_err(ctx, "tolerance must be >= 0"); return RAK_ERR_INVALID_ARGUMENT; }
  // every mode defaults to the CPU rules: the GPU rules' unclamped decrement lets R-MAT-like graphs
  // collapse into one community (as the reference GPU path does); they stay selectable
  r->rule = o->sketch_rule <= 0 ? 1 : o->sketch_rule;
  if (r->rule != 1 && r->rule != 2) { set_err(ctx, "sketch_rule must be -1, 0, 1 or 2"); return RAK_ERR_INVALID_ARGUMENT; }
  if (r->mode == RAK_MODE_SYNC && r->rule != 1) {
    set_err(ctx, "RAK_MODE_SYNC runs the CPU sketch rules (bit-exact with the reference CPU code)");
    return RAK_ERR_UNSUPPORTED;
  }
  // labels by vertex id by default (rak::default_label_order): with hashed ties (tie_break 2) id
  // labels no longer stall Misra-Gries runs on grid-numbered graphs, and on R-MAT they were faster
  // and never collapsed in repeated runs where the reference order collapsed in some; asynchronous
  // runs with one or two slots, whose sketches end on the last neighbour rather than on a tie, keep
  // the reference order against the stall
  r->order = o->label_order <= 0 ? rak::default_label_order(r->mode, r->slots) : o->label_order;
  if (r->order != 1 && r->order != 2) { set_err(ctx, "label_order must be -1, 0, 1 or 2"); return RAK_ERR_INVALID_ARGUMENT; }
  if (r->order == 2 && r->mode != RAK_MODE_ASYNC) {
    set_err(ctx, "the synchronous modes label vertices by id (bit-exact with the reference CPU code)");
    return RAK_ERR_UNSUPPORTED;
  }
  if (o->wait_timeout_ns < 0) { set_err(ctx, "wait_timeout_ns must be >= 0"); return RAK_ERR_INVALID_ARGUMENT; }
  // ties: hashed during the first iterations of asynchronous runs (measured: lattices +11% Q,
  // R-MAT and SBM unchanged or better); the reference's rule otherwise
  const int tie = o->tie_break <= 0 ? (r->mode == RAK_MODE_ASYNC && r->rule == 1 ? 2 : 1) : o->tie_break;
  if (tie != 1 && tie != 2) { set_err(ctx, "tie_break must be -1, 0, 1 or 2"); return RAK_ERR_INVALID_ARGUMENT; }
  if (tie == 2 && r->rule != 1) {
    set_err(ctx, "hashed ties apply to the CPU sketch rules (sketch_rule 1)");
    return RAK_ERR_UNSUPPORTED;
  }
  if (o->tie_iterations < 0) { set_err(ctx, "tie_iterations must be >= 0"); return RAK_ERR_INVALID_ARGUMENT; }
  r->tie_until = tie == 2 ? (o->tie_iterations > 0 ? o->tie_iterations : rak::DEFAULT_TIE_ITERATIONS) : 0;
  const int stg = o->edge_staging <= 0 ? rak::DEFAULT_EDGE_STAGING : o->edge_staging;
  if (stg != 1 && stg != 2) { set_err(ctx, "edge_staging must be -1, 0, 1 or 2"); return RAK_ERR_INVALID_ARGUMENT; }
  r->stage = stg == 1;
  if (o->max_blocks < 0) { set_err(ctx, "max_blocks must be >= 0"); return RAK_ERR_INVALID_ARGUMENT; }
  r->max_blocks = o->max_blocks;
  if (o->dense_pct > 100) { set_err(ctx, "dense_pct must be <= 100"); return RAK_ERR_INVALID_ARGUMENT; }
  r->dense_pct = o->dense_pct;
  // renumbered runs: the asynchronous default; the synchronous split mode on request (its results
  // are those of the graph as given, bit for bit, under the reference's tie rule); never the exact
  // synchronous mode
  if (o->renumber > 2) { set_err(ctx, "renumber must be -1, 0, 1 or 2"); return RAK_ERR_INVALID_ARGUMENT; }
  if (r->mode == RAK_MODE_SYNC || o->renumber == 2) r->renumber = 0;
  else if (o->renumber == 1) r->renumber = 2;
  else r->renumber = r->mode == RAK_MODE_ASYNC ? 1 : 0;
  r->timeout_ns = o->wait_timeout_ns > 0 ? (long long)o->wait_timeout_ns : rak::DEFAULT_WAIT_TIMEOUT_NS;
  r->start = o->start_iteration;
  r->validate = o->validate;
  r->modularity = o->compute_modularity;
  r->repeat = o->repeat < 1 ? 1 : o->repeat;
  r->ly.lane_max = o->lane_max > 0 ? o->lane_max : rak::DEFAULT_LANE_MAX;
  r->ly.hub_min = o->hub_min > 0 ? o->hub_min : rak::DEFAULT_HUB_MIN;
  r->ly.hub_chunk = o->hub_chunk > 0 ? o->hub_chunk : rak::DEFAULT_HUB_CHUNK;
  if (r->ly.lane_max > rak::MAX_LANE_MAX || r->ly.hub_min < r->ly.lane_max || r->ly.hub_chunk < 32) {
    set_err(ctx, "layout needs lane_max <= %lld, hub_min >= lane_max, hub_chunk >= 32",
            (long long)rak::MAX_LANE_MAX);
    return RAK_ERR_INVALID_ARGUMENT;
  }
  return RAK_OK;
}

// Batches (and the server's packed launches) label by vertex id unless the reference order is
// asked for: measured on the config-4 mix of R-MAT and SBM graphs, the reference order costs a
// batch about 9% modularity and 10% time, while single graphs need it against the pickless stall
// on grid-numbered ids.
void batch_default_order(const rak_options *o, Resolved *r) {
  if (!o || o->label_order <= 0) r->order = 1;
}

// Graph steps run one iteration on the caller's labels: an explicit request for the reference
// label order is refused rather than ignored.
rak_status ids_only(rak_ctx *ctx, const rak_options *o, Resolved *r) {
  if (o && o->label_order == 2) {
    set_err(ctx, "label_order 2 does not apply to rak_graph_step (labels are the caller's)");
    return RAK_ERR_UNSUPPORTED;
  }
  r->order = 1;
  return RAK_OK;
}

rak_status check_csr_shape(rak_ctx *ctx, const rak_csr *g) {
  if (!g) { set_err(ctx, "null csr"); return RAK_ERR_INVALID_ARGUMENT; }
  if (g->n < 0 || g->n >= (int64_t(1) << 31) || g->m < 0) { set_err(ctx, "csr sizes out of range (n=%lld m=%lld)", (long long)g->n, (long long)g->m); return RAK_ERR_INVALID_ARGUMENT; }
  if (g->offset_bits != 32 && g->offset_bits != 64) { set_err(ctx, "offset_bits must be 32 or 64"); return RAK_ERR_INVALID_ARGUMENT; }
  if (g->offset_bits == 32 && g->m > int64_t(std::numeric_limits<int32_t>::max())) { set_err(ctx, "m too large for 32-bit offsets"); return RAK_ERR_INVALID_ARGUMENT; }
  if (g->location != RAK_HOST && g->location != RAK_DEVICE) { set_err(ctx, "bad location"); return RAK_ERR_INVALID_ARGUMENT; }
  if (!g->offsets || (g->m > 0 && !g->targets)) { set_err(ctx, "null csr arrays"); return RAK_ERR_INVALID_ARGUMENT; }
  return RAK_OK;
}

// Branch-free inside blocks of 64K entries so that the scans vectorise; the target scan of a
// large graph is split over OpenMP threads.
template <class O>
rak_status validate_host_t(const O *off, const uint32_t *tgt, int64_t n, int64_t m) {
  if (int64_t(off[0]) != 0 || int64_t(off[n]) != m) return RAK_ERR_INVALID_CSR;
  constexpr int64_t BLK = 1 << 16;
  for (int64_t b = 0; b < n; b += BLK) {
    const int64_t e = std::min(n, b + BLK);
    unsigned bad = 0;
    for (int64_t u = b; u < e; ++u) bad |= unsigned(off[u] > off[u + 1]);
    if (bad) return RAK_ERR_INVALID_CSR;
  }
  if (n >= (int64_t(1) << 32)) return RAK_OK;  // every 32-bit target is in range
  const uint32_t lim = uint32_t(n);
  const int64_t nblk = (m + BLK - 1) / BLK;
  unsigned bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad) if (m >= (int64_t(1) << 21))
  for (int64_t k = 0; k < nblk; ++k) {
    const int64_t b = k * BLK, e = std::min(m, b + BLK);
    unsigned blk = 0;
    for (int64_t i = b; i < e; ++i) blk |= unsigned(tgt[i] >= lim);
    bad |= blk;
  }
  return bad ? RAK_ERR_INVALID_CSR : RAK_OK;
}

int nkeys_of(const Layout &ly) { return int(6 + ly.lane_max + 1); }

// Region sizes, item counts and chunk table from the key histogram and split-vertex degrees.
void regions_from(const std::vector<unsigned long long> &hist, const Layout &ly, int64_t nchunks, int sms,
                  rak::Regions *rg) {
  int64_t cnt[rak::NREG] = {};
  for (int k = 0; k < 6; ++k) cnt[k] = int64_t(hist[k]);
  for (int64_t k = 6; k < 6 + ly.lane_max; ++k) cnt[rak::REG_LANE] += int64_t(hist[k]);
  rg->lane_item = rak::lane_item_for(cnt[rak::REG_LANE], int64_t(sms) * rak::LPA_WARPS_PER_SM);
  int64_t v = 0, it = 0;
  for (int r = 0; r < rak::NREG; ++r) {
    rg->vbegin[r] = v;
    rg->vcount[r] = cnt[r];
    v += cnt[r];
    rg->ibegin[r] = it;
    it += rak::region_items(r, cnt[r], nchunks, rg->lane_item);
  }
  rg->ibegin[rak::NREG] = it;
}

rak_status build_plan(rak_ctx *ctx, rak_graph *gr, const Layout &ly, Tracker *tr) {
  cudaStream_t st = ctx->stream;
  gr->ly = ly;
  const int64_t n = gr->n;
  const int nk = nkeys_of(ly);
  Events ev;
  cudaEventRecord(ev.e[0], st);
  const size_t n4 = size_t(std::max<int64_t>(n, 1)) * 4;
  RAK_TRY(ctx, ensure(gr->p_order, n4));
  RAK_TRY(ctx, ensure(gr->p_keys, n4));
  RAK_TRY(ctx, ensure(gr->p_keys2, n4));
  RAK_TRY(ctx, ensure(gr->p_vids, n4));
  RAK_TRY(ctx, ensure(gr->p_hist, size_t(nk) * 8));
  gr->order = gr->p_order.as<uint32_t>();
  if (tr) tr->add(n4 * 4 + size_t(nk) * 8);
  RAK_TRY(ctx, cudaMemsetAsync(gr->p_hist.p, 0, size_t(nk) * 8, st));
  std::vector<unsigned long long> h(size_t(nk), 0);
  if (n > 0) {
    RAK_TRY(ctx, rak::launch_plan_keys(gr->off, gr->off64, n, ly, gr->p_keys.as<uint32_t>(), gr->p_vids.as<uint32_t>(),
                                       gr->p_hist.as<unsigned long long>(), nk, st));
    int end_bit = 1;
    while ((1 << end_bit) < nk) ++end_bit;
    size_t tb = 0;
    RAK_TRY(ctx, rak::plan_sort(gr->p_keys.as<uint32_t>(), gr->p_keys2.as<uint32_t>(), gr->p_vids.as<uint32_t>(),
                                gr->order, n, end_bit, nullptr, &tb, st));
    RAK_TRY(ctx, ensure(gr->p_temp, tb));
    if (tr) tr->add(gr->p_temp.bytes);
    RAK_TRY(ctx, rak::plan_sort(gr->p_keys.as<uint32_t>(), gr->p_keys2.as<uint32_t>(), gr->p_vids.as<uint32_t>(),
                                gr->order, n, end_bit, gr->p_temp.p, &tb, st));
    RAK_TRY(ctx, cudaMemcpyAsync(h.data(), gr->p_hist.p, size_t(nk) * 8, cudaMemcpyDeviceToHost, st));
    RAK_TRY(ctx, cudaStreamSynchronize(st));
  }
  gr->nhub = int64_t(h.empty() ? 0 : h[0]);
  gr->nchunks = 0;
  gr->hub_first = nullptr;
  gr->chunk_hub = nullptr;
  std::vector<int64_t> first(size_t(gr->nhub) + 1, 0);
  if (gr->nhub > 0) {
    RAK_TRY(ctx, ensure(gr->p_deg, size_t(gr->nhub) * 8));
    RAK_TRY(ctx, rak::launch_hub_degrees(gr->off, gr->off64, gr->order, gr->nhub, gr->p_deg.as<int64_t>(), st));
    std::vector<int64_t> hd(size_t(gr->nhub));
    RAK_TRY(ctx, cudaMemcpyAsync(hd.data(), gr->p_deg.p, size_t(gr->nhub) * 8, cudaMemcpyDeviceToHost, st));
    RAK_TRY(ctx, cudaStreamSynchronize(st));
    for (int64_t i = 0; i < gr->nhub; ++i) first[i + 1] = first[i] + (hd[i] + ly.hub_chunk - 1) / ly.hub_chunk;
    gr->nchunks = first[gr->nhub];
    std::vector<uint32_t> ch(size_t(gr->nchunks));
    for (int64_t i = 0; i < gr->nhub; ++i)
      for (int64_t c = first[i]; c < first[i + 1]; ++c) ch[c] = uint32_t(i);
    RAK_TRY(ctx, ensure(gr->p_hub_first, first.size() * 8));
    RAK_TRY(ctx, ensure(gr->p_chunk_hub, ch.size() * 4));
    gr->hub_first = gr->p_hub_first.as<int64_t>();
    gr->chunk_hub = gr->p_chunk_hub.as<uint32_t>();
    if (tr) tr->add(first.size() * 8 + ch.size() * 4);
    RAK_TRY(ctx, cudaMemcpyAsync(gr->hub_first, first.data(), first.size() * 8, cudaMemcpyHostToDevice, st));
    RAK_TRY(ctx, cudaMemcpyAsync(gr->chunk_hub, ch.data(), ch.size() * 4, cudaMemcpyHostToDevice, st));
  }
  gr->plan_bytes = gr->p_order.bytes + gr->p_hub_first.bytes + gr->p_chunk_hub.bytes;
  regions_from(h, ly, gr->nchunks, ctx->sms, &gr->rg);
  cudaEventRecord(ev.e[1], st);
  RAK_TRY(ctx, cudaStreamSynchronize(st));
  gr->plan_ms = ev.ms(0, 1);
  return RAK_OK;
}

bool same_layout(const Layout &a, const Layout &b) {
  return a.lane_max == b.lane_max && a.hub_min == b.hub_min && a.hub_chunk == b.hub_chunk;
}

rak_status graph_create(rak_ctx *ctx, const rak_csr *g, const Resolved &r, Tracker *tr, rak_graph **out) {
  RAK_CHECK(check_csr_shape(ctx, g));
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  auto *gr = new (std::nothrow) rak_graph();
  if (!gr) return RAK_ERR_OUT_OF_MEMORY;
  gr->ctx = ctx;
  gr->device = ctx->device;
  gr->n = g->n;
  gr->m = g->m;
  gr->off64 = g->offset_bits == 64;
  const size_t ob = size_t(g->n + 1) * (gr->off64 ? 8 : 4);
  auto fail = [&](rak_status s) { rak_graph_destroy(gr); return s; };
  if (g->location == RAK_DEVICE) {
    gr->off = g->offsets;
    gr->tgt = g->targets;
    gr->wt = g->weights;
    gr->ref_bytes = ob + uint64_t(g->m) * 4 * (g->weights ? 2 : 1);
    if (tr) tr->add(gr->ref_bytes);
  } else {
    // a host graph is checked on the device once uploaded (below): the copies touch only the
    // n + 1 offsets and m edges it declares, and the device reads it ~100x faster than the host
    gr->owns = true;
    Events ev;
    void *po = nullptr, *pt = nullptr, *pw = nullptr;
    gr->arrays_pooled = rak_host_detail::thread_pool().pool != nullptr;
    cudaError_t e = rak_host_detail::dev_alloc(&po, ob, &gr->arrays_fs);
    if (e == cudaSuccess) e = rak_host_detail::dev_alloc(&pt, size_t(std::max<int64_t>(g->m, 1)) * 4, &gr->arrays_fs);
    if (e == cudaSuccess && g->weights)
      e = rak_host_detail::dev_alloc(&pw, size_t(std::max<int64_t>(g->m, 1)) * 4, &gr->arrays_fs);
    gr->off = po; gr->tgt = static_cast<uint32_t *>(pt); gr->wt = static_cast<float *>(pw);
    gr->off_cap = ob;
    gr->tgt_cap = size_t(std::max<int64_t>(g->m, 1)) * 4;
    gr->wt_cap = g->weights ? gr->tgt_cap : 0;
    gr->wt_alloc = pw;
    if (e != cudaSuccess) return fail(from_cuda(ctx, e, "cudaMalloc(graph)"));
    gr->graph_bytes = ob + size_t(std::max<int64_t>(g->m, 1)) * 4 * (g->weights ? 2 : 1);
    if (tr) tr->add(gr->graph_bytes);
    cudaEventRecord(ev.e[0], ctx->stream);
    e = cudaMemcpyAsync(po, g->offsets, ob, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && g->m > 0) e = cudaMemcpyAsync(pt, g->targets, size_t(g->m) * 4, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && g->weights && g->m > 0) e = cudaMemcpyAsync(pw, g->weights, size_t(g->m) * 4, cudaMemcpyHostToDevice, ctx->stream);
    cudaEventRecord(ev.e[1], ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail(from_cuda(ctx, e, "copy graph to device"));
    gr->h2d_ms = ev.ms(0, 1);
  }
  if (r.validate) {
    DevBuf bad;
    cudaError_t e = bad.alloc(4, tr);
    unsigned int hbad = 0;
    if (e == cudaSuccess) e = cudaMemsetAsync(bad.p, 0, 4, ctx->stream);
    if (e == cudaSuccess) e = rak::launch_validate(gr->off, gr->off64, gr->tgt, gr->n, gr->m, bad.as<unsigned int>(), ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad.p, 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail(from_cuda(ctx, e, "validate csr"));
    if (hbad) { set_err(ctx, "invalid CSR (device check: %s)", hbad & 2 ? "target out of range" : "offsets"); return fail(RAK_ERR_INVALID_CSR); }
  }
  rak_status s = build_plan(ctx, gr, r.ly, tr);
  if (s != RAK_OK) return fail(s);
  *out = gr;
  return RAK_OK;
}

// The renumbered copy of a resident graph (rak_renumber.cu), for the graph's current layout.
rak_status ensure_renumbered(rak_ctx *ctx, rak_graph *gr, Tracker *tr) {
  if (gr->rn_ready && same_layout(gr->rn_ly, gr->ly)) return RAK_OK;
  cudaStream_t st = ctx->stream;
  const int64_t n = gr->n, m = gr->m;
  const size_t ob = gr->off64 ? 8 : 4;
  Events ev;
  cudaEventRecord(ev.e[0], st);
  RAK_TRY(ctx, ensure(gr->rn_inv, size_t(n) * 4));
  RAK_TRY(ctx, ensure(gr->rn_ident, size_t(n) * 4));
  RAK_TRY(ctx, ensure(gr->rn_off, size_t(n + 1) * ob));
  RAK_TRY(ctx, ensure(gr->rn_tgt, size_t(m) * 4));
  if (gr->wt) RAK_TRY(ctx, ensure(gr->rn_wt, size_t(m) * 4));
  if (tr) tr->add(gr->rn_bytes());   // counted while the build's own space is held
  DevBuf deg, temp;
  RAK_TRY(ctx, deg.alloc(size_t(n + 1) * ob, tr));
  size_t tb = 0;
  RAK_TRY(ctx, rak::renumber_graph(gr->off, gr->off64, gr->tgt, gr->wt, gr->order, n, gr->rg.vbegin[rak::REG_LANE],
                                   gr->rn_inv.as<uint32_t>(), deg.p, gr->rn_off.p, gr->rn_tgt.as<uint32_t>(),
                                   gr->wt ? gr->rn_wt.as<float>() : nullptr, gr->rn_ident.as<uint32_t>(), nullptr,
                                   &tb, st));
  RAK_TRY(ctx, temp.alloc(tb, tr));
  RAK_TRY(ctx, rak::renumber_graph(gr->off, gr->off64, gr->tgt, gr->wt, gr->order, n, gr->rg.vbegin[rak::REG_LANE],
                                   gr->rn_inv.as<uint32_t>(), deg.p, gr->rn_off.p, gr->rn_tgt.as<uint32_t>(),
                                   gr->wt ? gr->rn_wt.as<float>() : nullptr, gr->rn_ident.as<uint32_t>(), temp.p,
                                   &tb, st));
  cudaEventRecord(ev.e[1], st);
  RAK_TRY(ctx, cudaStreamSynchronize(st));
  if (tr) tr->sub(gr->rn_bytes());
  gr->plan_ms += ev.ms(0, 1);
  gr->rn_ready = true;
  gr->rn_ly = gr->ly;
  return RAK_OK;
}

// The complete run on a resident graph; labels end up in vcom0 (caller-provided, n entries).
rak_status run_resident(rak_ctx *ctx, rak_graph *gr, const uint32_t *q, const uint8_t *flags,
                        const Resolved &r, uint32_t *vcom0, Tracker *tr, rak_result *res) {
  cudaStream_t st = ctx->stream;
  if (!same_layout(gr->ly, r.ly)) RAK_CHECK(build_plan(ctx, gr, r.ly, tr));
  const int64_t n = gr->n;
  const bool sync = r.mode != RAK_MODE_ASYNC;
  const int iters = std::max(r.iters, 1);
  RunBufs &b = gr->bufs;
  RAK_TRY(ctx, ensure(b.aff0, size_t(n) + 16));
  if (sync) {
    RAK_TRY(ctx, ensure(b.vcom1, size_t(n) * 4 + 16));
    RAK_TRY(ctx, ensure(b.aff1, size_t(n) + 16));
  }
  const size_t nh = size_t(std::max<int64_t>(gr->nhub, 1)), nc = size_t(std::max<int64_t>(gr->nchunks, 1));
  RAK_TRY(ctx, ensure(b.arrive, nh * 4));
  RAK_TRY(ctx, ensure(b.claim, nh * 4));
  RAK_TRY(ctx, ensure(b.moved, nh * 4));
  RAK_TRY(ctx, ensure(b.skk, nc * size_t(r.slots) * 4));
  RAK_TRY(ctx, ensure(b.skw, nc * size_t(r.slots) * 4));
  RAK_TRY(ctx, ensure(b.stats, size_t(iters) * rak::STATS_STRIDE * 8));
  RAK_TRY(ctx, ensure(b.rs, sizeof(rak::RunStateHost)));
  // asynchronous id-label runs work on the graph renumbered in work order (rak_renumber.cu)
  // by default only resident graphs, run again and again, pay for the copy (R-MAT scale 27: about
  // 80 ms once, 26 ms less per run), and only large dense ones: on a sparse R-MAT (scale 25, average
  // degree 8) the copy made runs slower (8.4 -> 10.6 ms), on the 2^25 lattice 4% faster
  bool renum = r.iters > 0 && n > 0 &&
               (r.renumber == 2 || (r.renumber == 1 && !r.one_shot && rak::mark_test_for(n, gr->m)));
  if (renum && r.renumber == 1 && !(gr->rn_ready && same_layout(gr->rn_ly, gr->ly))) {
    // by default the copy is only made when it fits beside what the device holds, with 1 GiB to
    // spare; otherwise the run works on the graph as given
    size_t free_b = 0, total_b = 0;
    const size_t need = size_t(n) * (gr->off64 ? 8 : 4) * 2 + size_t(n) * 12 + size_t(gr->m) * (gr->wt ? 8 : 4) +
                        (size_t(1) << 30);
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { cudaGetLastError(); free_b = 0; }
    if (free_b < need) renum = false;
  }
  if (renum) {
    RAK_TRY(ctx, ensure(b.lab, size_t(n) * 4));
    RAK_CHECK(ensure_renumbered(ctx, gr, tr));
    if (tr) tr->add(gr->rn_bytes());
  }
  if (tr) tr->add(b.bytes());

  rak::LpaArgs a{};
  a.off = gr->off; a.tgt = gr->tgt; a.wt = gr->wt; a.n = n;
  a.order = gr->order; a.rg = gr->rg;
  a.chunk_hub = gr->chunk_hub; a.hub_first = gr->hub_first; a.hub_chunk = gr->ly.hub_chunk; a.nchunks = gr->nchunks;
  a.vcom0 = vcom0; a.vcom1 = b.vcom1.as<uint32_t>(); a.aff0 = b.aff0.as<uint8_t>(); a.aff1 = b.aff1.as<uint8_t>();
  a.hub_arrive = b.arrive.as<uint32_t>(); a.hub_claim = b.claim.as<uint32_t>(); a.hub_moved = b.moved.as<int32_t>();
  a.sk_keys = b.skk.as<uint32_t>(); a.sk_wts = b.skw.as<float>();
  a.stats = b.stats.as<unsigned long long>(); a.rs = b.rs.p;
  a.iters = r.iters; a.start_iter = r.start; a.tolerance = r.tol; a.pickless_step = r.pickless;
  a.check_on_pickless = r.check_on_pickless; a.rescan = r.rescan; a.mark_test = rak::mark_test_for(a.n, gr->m); a.gpu_rule = r.rule == 2; a.timeout_ns = r.timeout_ns; a.tie_until = r.tie_until; a.stage = r.stage; a.grid_cap = r.max_blocks;
  a.dense_moved_edges = rak::dense_threshold(r.mode, r.dense_pct, gr->m);
  if (renum) {
    a.off = gr->rn_off.p; a.tgt = gr->rn_tgt.as<uint32_t>(); a.wt = gr->wt ? gr->rn_wt.as<float>() : nullptr;
    a.order = gr->rn_ident.as<uint32_t>();
    a.vcom0 = b.lab.as<uint32_t>();
  }

  // the kernel's module is loaded here, not inside the timed region
  if (r.iters > 0) RAK_TRY(ctx, rak::prepare_lpa(r.slots, r.mode, gr->off64, gr->wt == nullptr, false, r.stage));
  // Labels as positions in the reference GPU path's vertex order (inc/rakLowmemCuda.hxx:563,
  // 591-592), so that its pickless rule compares the same label order; turned back into vertex ids
  // after the run. The order depends on degrees only: built once per graph.
  const bool ref_labels = r.order == 2 && n > 0;
  if (ref_labels && !gr->ref_ready) {
    DevBuf scratch;
    RAK_TRY(ctx, ensure(gr->ref_ks, size_t(n) * 4));
    RAK_TRY(ctx, ensure(gr->ref_pos, size_t(n) * 4));
    RAK_TRY(ctx, scratch.alloc(rak::ref_order_scratch_bytes(n, 1), nullptr));
    RAK_TRY(ctx, rak::ref_order(gr->off, gr->off64, n, nullptr, nullptr, 0, gr->ref_ks.as<uint32_t>(),
                                gr->ref_pos.as<uint32_t>(), scratch.p, st));
    RAK_TRY(ctx, cudaStreamSynchronize(st));
    gr->ref_ready = true;
  }
  if (ref_labels && tr) tr->add(gr->ref_ks.bytes + gr->ref_pos.bytes);
  Events ev;
  float t_init = 0, t_mark = 0, t_all = 0, t_loop = 0;
  rak::RunStateHost hs{};
  std::vector<unsigned long long> stats(size_t(iters) * rak::STATS_STRIDE, 0);
  for (int rep = 0; rep < r.repeat; ++rep) {
    RAK_TRY(ctx, cudaMemsetAsync(b.arrive.p, 0, b.arrive.bytes, st));
    RAK_TRY(ctx, cudaMemsetAsync(b.claim.p, 0, b.claim.bytes, st));
    RAK_TRY(ctx, cudaMemsetAsync(b.moved.p, 0xFF, b.moved.bytes, st));
    RAK_TRY(ctx, cudaMemsetAsync(b.stats.p, 0, b.stats.bytes, st));
    RAK_TRY(ctx, cudaMemsetAsync(b.rs.p, 0, b.rs.bytes, st));
    cudaEventRecord(ev.e[0], st);
    if (renum) {
      RAK_TRY(ctx, rak::launch_renumbered_init(gr->order, q, ref_labels ? gr->ref_pos.as<uint32_t>() : nullptr, flags,
                                               n, a.vcom0, a.aff0, st));
      if (sync) {
        RAK_TRY(ctx, cudaMemcpyAsync(a.vcom1, a.vcom0, size_t(n) * 4, cudaMemcpyDeviceToDevice, st));
        RAK_TRY(ctx, cudaMemsetAsync(a.aff1, 0, size_t(n), st));
      }
    } else if (ref_labels) RAK_TRY(ctx, rak::launch_init_mapped(vcom0, q, gr->ref_pos.as<uint32_t>(), n, st));
    else RAK_TRY(ctx, rak::launch_init(vcom0, sync ? a.vcom1 : nullptr, q, n, st));
    cudaEventRecord(ev.e[1], st);
    if (!renum) RAK_TRY(ctx, rak::launch_init_flags(a.aff0, sync ? a.aff1 : nullptr, flags, n, st));
    cudaEventRecord(ev.e[2], st);
    if (r.iters > 0) {
      int grid = 0;
      RAK_TRY(ctx, rak::launch_lpa(a, r.slots, r.mode, gr->off64, st, &grid));
    }
    cudaEventRecord(ev.e[3], st);
    RAK_TRY(ctx, cudaStreamSynchronize(st));
    t_init += ev.ms(0, 1);
    t_mark += ev.ms(1, 2);
    t_loop += ev.ms(2, 3);
    t_all += ev.ms(0, 3);
  }
  RAK_TRY(ctx, cudaMemcpyAsync(&hs, b.rs.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
  RAK_TRY(ctx, cudaMemcpyAsync(stats.data(), b.stats.p, stats.size() * 8, cudaMemcpyDeviceToHost, st));
  RAK_TRY(ctx, cudaStreamSynchronize(st));
  if (hs.error) {
    set_err(ctx, "device-side wait gave up (status %u)", hs.error);
    return rak_status(hs.error);
  }
  const int done = r.iters > 0 ? int(hs.iterations) : 0;
  if (sync && (done & 1)) RAK_TRY(ctx, cudaMemcpyAsync(a.vcom0, a.vcom1, size_t(n) * 4, cudaMemcpyDeviceToDevice, st));
  if (renum) RAK_TRY(ctx, rak::launch_renumbered_gather(b.lab.as<uint32_t>(), gr->rn_inv.as<uint32_t>(), n, vcom0, st));
  if (ref_labels) RAK_TRY(ctx, rak::launch_labels_to_ids(vcom0, gr->ref_ks.as<uint32_t>(), n, st));
  RAK_TRY(ctx, cudaStreamSynchronize(st));
  if (res) {
    res->iterations = done;
    res->time_ms = t_all / float(r.repeat);
    res->initialization_time_ms = t_init / float(r.repeat);
    res->marking_time_ms = t_mark / float(r.repeat);
    res->loop_ms = t_loop / float(r.repeat);
    res->traversed_edges = res->processed_vertices = res->moved_vertices = res->moved_edges = res->marked_edges = 0;
    res->dense_iterations = 0;
    for (int i = 0; i < done; ++i) {
      const unsigned long long *st_i = &stats[size_t(i) * rak::STATS_STRIDE];
      res->traversed_edges += st_i[rak::STAT_EDGES];
      res->processed_vertices += st_i[rak::STAT_PROCESSED];
      res->moved_vertices += st_i[rak::STAT_CHANGED];
      res->moved_edges += st_i[rak::STAT_MOVED_EDGES];
      if (st_i[rak::STAT_PHASE] & 1ull) res->dense_iterations += 1;
      else res->marked_edges += st_i[rak::STAT_MOVED_EDGES];
    }
    res->changed_last = done > 0 ? stats[size_t(done - 1) * rak::STATS_STRIDE + rak::STAT_CHANGED] : 0;
    res->memory_gb = float(double(b.bytes() + size_t(n) * 4 + gr->plan_bytes + (renum ? gr->rn_bytes() : 0)) /
                           (1024.0 * 1024.0 * 1024.0));
    res->plan_ms = gr->plan_ms;
  }
  return RAK_OK;
}

rak_status modularity_dev(rak_ctx *ctx, const void *off, bool off64, const uint32_t *tgt, const float *wt, int64_t n,
                          const uint32_t *labels, Tracker *tr, double *q) {
  DevBuf ctot, sums;
  RAK_TRY(ctx, ctot.alloc(size_t(std::max<int64_t>(n, 1)) * 8, tr));
  RAK_TRY(ctx, sums.alloc(4 * 8, tr));
  RAK_TRY(ctx, cudaMemsetAsync(ctot.p, 0, ctot.bytes, ctx->stream));
  RAK_TRY(ctx, cudaMemsetAsync(sums.p, 0, sums.bytes, ctx->stream));
  double h[4] = {0, 0, 0, 0};
  if (n > 0) RAK_TRY(ctx, rak::launch_modularity(off, off64, tgt, wt, n, labels, ctot.as<double>(), sums.as<double>(), ctx->stream));
  RAK_TRY(ctx, cudaMemcpyAsync(h, sums.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (h[3] > 0) { set_err(ctx, "membership holds labels >= n"); return RAK_ERR_INVALID_ARGUMENT; }
  *q = h[1] > 0 ? h[0] / h[1] - h[2] / (h[1] * h[1]) : 0.0;
  return RAK_OK;
}

}  // namespace

extern "C" {

int rak_abi_version(void) { return RAK_ABI_VERSION; }

const char *rak_status_string(rak_status s) {
  switch (s) {
    case RAK_OK: return "ok";
    case RAK_ERR_INVALID_ARGUMENT: return "invalid argument";
    case RAK_ERR_INVALID_CSR: return "invalid CSR";
    case RAK_ERR_OUT_OF_MEMORY: return "out of memory";
    case RAK_ERR_CUDA: return "CUDA error";
    case RAK_ERR_TIMEOUT: return "device-side wait timed out";
    case RAK_ERR_NO_DEVICE: return "no usable CUDA device";
    case RAK_ERR_UNSUPPORTED: return "unsupported option combination";
    case RAK_ERR_BUSY: return "busy";
  }
  return "unknown status";
}

void rak_options_default(rak_options *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->repeat = 1;
  o->tolerance = 0.05;
  o->max_iterations = 20;
  o->slots = 8;
  o->mode = RAK_MODE_ASYNC;
  o->rescan = -1;
  o->pickless_step = -1;
  o->check_on_pickless = -1;
  o->validate = 1;
  o->sketch_rule = -1;
  o->label_order = -1;
}

rak_status rak_ctx_create(int device, rak_ctx **out) {
  if (!out) return RAK_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || device < 0 || device >= count) { cudaGetLastError(); return RAK_ERR_NO_DEVICE; }
  cudaDeviceProp p{};
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess || p.major != 10) return RAK_ERR_NO_DEVICE;
  auto *ctx = new (std::nothrow) rak_ctx();
  if (!ctx) return RAK_ERR_OUT_OF_MEMORY;
  ctx->device = device;
  ctx->sms = p.multiProcessorCount;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return RAK_ERR_CUDA;
  }
  ctx->stream = ctx->own;
  *out = ctx;
  return RAK_OK;
}

rak_status rak_ctx_destroy(rak_ctx *ctx) {
  if (!ctx) return RAK_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  if (ctx->pool) {
    cudaDeviceSynchronize();
    cudaMemPoolDestroy(ctx->pool);
  }
  if (ctx->own) cudaStreamDestroy(ctx->own);
  delete ctx;
  return RAK_OK;
}

rak_status rak_ctx_set_stream(rak_ctx *ctx, void *stream) {
  if (!ctx) return RAK_ERR_INVALID_ARGUMENT;
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own;
  return RAK_OK;
}

rak_status rak_ctx_set_memory_keep(rak_ctx *ctx, uint64_t bytes) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx) return RAK_ERR_INVALID_ARGUMENT;
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  if (!ctx->pool) {
    if (bytes == 0) return RAK_OK;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx->device;
    RAK_TRY(ctx, cudaMemPoolCreate(&ctx->pool, &props));
  }
  uint64_t keep = bytes;
  RAK_TRY(ctx, cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  if (bytes == 0) {  // back to cudaMalloc/cudaFree: a pool that keeps nothing re-maps on every call
    RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    RAK_TRY(ctx, cudaMemPoolTrimTo(ctx->pool, 0));
  }
  ctx->keep = bytes;
  return RAK_OK;
}

const char *rak_ctx_last_error(const rak_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

rak_status rak_graph_create(rak_ctx *ctx, const rak_csr *g, const rak_options *o, rak_graph **out) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !out) return RAK_ERR_INVALID_ARGUMENT;
  Resolved r;
  RAK_CHECK(resolve(ctx, o, &r));
  return graph_create(ctx, g, r, nullptr, out);
}

rak_status rak_graph_destroy(rak_graph *gr) {
  if (!gr) return RAK_ERR_INVALID_ARGUMENT;
  cudaSetDevice(gr->device);
  if (gr->owns) {
    rak_host_detail::dev_free(const_cast<void *>(gr->off), gr->arrays_pooled, gr->arrays_fs);
    rak_host_detail::dev_free(const_cast<uint32_t *>(gr->tgt), gr->arrays_pooled, gr->arrays_fs);
    rak_host_detail::dev_free(gr->wt_alloc, gr->arrays_pooled, gr->arrays_fs);
  }
  delete gr;
  return RAK_OK;
}

uint64_t rak_graph_device_bytes(const rak_graph *gr) {
  return gr ? gr->graph_bytes + gr->plan_bytes + gr->rn_bytes() : 0;
}

rak_status rak_graph_run(rak_ctx *ctx, rak_graph *gr, const uint32_t *q, const rak_options *o,
                         uint32_t *membership, rak_result *res) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !gr || !membership) return RAK_ERR_INVALID_ARGUMENT;
  Resolved r;
  RAK_CHECK(resolve(ctx, o, &r));
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  Tracker tr;
  tr.add(gr->graph_bytes + gr->ref_bytes + gr->plan_bytes);
  rak_result tmp{};
  rak_result *rr = res ? res : &tmp;
  std::memset(rr, 0, sizeof(*rr));
  rr->modularity = std::numeric_limits<double>::quiet_NaN();
  RAK_CHECK(run_resident(ctx, gr, q, o ? o->initial_flags : nullptr, r, membership, &tr, rr));
  if (r.modularity)
    RAK_CHECK(modularity_dev(ctx, gr->off, gr->off64, gr->tgt, gr->wt, gr->n, membership, &tr, &rr->modularity));
  rr->peak_device_bytes = tr.peak + size_t(gr->n) * 4;
  return RAK_OK;
}

rak_status rak_lowmem_cuda(rak_ctx *ctx, const rak_csr *g, const uint32_t *q, const rak_options *o,
                           uint32_t *membership, rak_result *res) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !g || !membership) return RAK_ERR_INVALID_ARGUMENT;
  Resolved r;
  RAK_CHECK(resolve(ctx, o, &r));
  r.one_shot = true;   // the graph lives for this call only
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  rak_result tmp{};
  rak_result *rr = res ? res : &tmp;
  std::memset(rr, 0, sizeof(*rr));
  rr->modularity = std::numeric_limits<double>::quiet_NaN();
  // with a context pool, this call's buffers are stream-ordered allocations from it (kept mapped
  // between calls up to the pool's threshold); otherwise cudaMalloc/cudaFree
  rak_host_detail::PoolScope scope(ctx->keep > 0 ? ctx->pool : nullptr, ctx->stream);
  Tracker tr;
  rak_graph *gr = nullptr;
  RAK_CHECK(graph_create(ctx, g, r, &tr, &gr));
  struct Guard { rak_graph *g; ~Guard() { rak_graph_destroy(g); } } guard{gr};
  const int64_t n = g->n;
  const uint8_t *flags = o ? o->initial_flags : nullptr;
  rr->h2d_ms = gr->h2d_ms;
  if (g->location == RAK_DEVICE) {
    RAK_CHECK(run_resident(ctx, gr, q, flags, r, membership, &tr, rr));
    if (r.modularity) RAK_CHECK(modularity_dev(ctx, gr->off, gr->off64, gr->tgt, gr->wt, n, membership, &tr, &rr->modularity));
    rr->peak_device_bytes = tr.peak;
    return RAK_OK;
  }
  DevBuf labels, qd, fd;
  RAK_TRY(ctx, labels.alloc(size_t(n) * 4 + 16, &tr));
  Events ev;
  cudaEventRecord(ev.e[0], ctx->stream);
  if (q) {
    RAK_TRY(ctx, qd.alloc(size_t(n) * 4 + 16, &tr));
    RAK_TRY(ctx, cudaMemcpyAsync(qd.p, q, size_t(n) * 4, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (flags) {
    RAK_TRY(ctx, fd.alloc(size_t(n) + 16, &tr));
    RAK_TRY(ctx, cudaMemcpyAsync(fd.p, flags, size_t(n), cudaMemcpyHostToDevice, ctx->stream));
  }
  cudaEventRecord(ev.e[1], ctx->stream);
  RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  rr->h2d_ms += ev.ms(0, 1);
  RAK_CHECK(run_resident(ctx, gr, qd.as<uint32_t>(), fd.as<uint8_t>(), r, labels.as<uint32_t>(), &tr, rr));
  if (r.modularity) RAK_CHECK(modularity_dev(ctx, gr->off, gr->off64, gr->tgt, gr->wt, n, labels.as<uint32_t>(), &tr, &rr->modularity));
  cudaEventRecord(ev.e[2], ctx->stream);
  RAK_TRY(ctx, cudaMemcpyAsync(membership, labels.p, size_t(n) * 4, cudaMemcpyDeviceToHost, ctx->stream));
  cudaEventRecord(ev.e[3], ctx->stream);
  RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  rr->d2h_ms = ev.ms(2, 3);
  rr->peak_device_bytes = tr.peak;
  return RAK_OK;
}

rak_status rak_graph_step(rak_ctx *ctx, rak_graph *gr, const rak_options *o, int iteration,
                          const uint32_t *vcom_prev, const uint8_t *aff_prev, uint32_t *vcom_next,
                          uint8_t *aff_next, uint64_t *changed) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !gr || !vcom_prev || !aff_prev || !vcom_next || !aff_next) return RAK_ERR_INVALID_ARGUMENT;
  Resolved r;
  RAK_CHECK(resolve(ctx, o, &r));
  RAK_CHECK(ids_only(ctx, o, &r));
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  if (!same_layout(gr->ly, r.ly)) RAK_CHECK(build_plan(ctx, gr, r.ly, nullptr));
  cudaStream_t st = ctx->stream;
  const int64_t n = gr->n;
  const bool sync = r.mode != RAK_MODE_ASYNC;
  RunBufs b;
  const size_t nh = size_t(std::max<int64_t>(gr->nhub, 1)), nc = size_t(std::max<int64_t>(gr->nchunks, 1));
  RAK_TRY(ctx, b.arrive.alloc(nh * 4, nullptr));
  RAK_TRY(ctx, b.claim.alloc(nh * 4, nullptr));
  RAK_TRY(ctx, b.moved.alloc(nh * 4, nullptr));
  RAK_TRY(ctx, b.skk.alloc(nc * size_t(r.slots) * 4, nullptr));
  RAK_TRY(ctx, b.skw.alloc(nc * size_t(r.slots) * 4, nullptr));
  RAK_TRY(ctx, b.stats.alloc(rak::STATS_STRIDE * 8, nullptr));
  RAK_TRY(ctx, b.rs.alloc(sizeof(rak::RunStateHost), nullptr));
  RAK_TRY(ctx, cudaMemsetAsync(b.arrive.p, 0, b.arrive.bytes, st));
  RAK_TRY(ctx, cudaMemsetAsync(b.claim.p, 0, b.claim.bytes, st));
  RAK_TRY(ctx, cudaMemsetAsync(b.moved.p, 0xFF, b.moved.bytes, st));
  RAK_TRY(ctx, cudaMemsetAsync(b.stats.p, 0, b.stats.bytes, st));
  RAK_TRY(ctx, cudaMemsetAsync(b.rs.p, 0, b.rs.bytes, st));
  if (vcom_next != vcom_prev) RAK_TRY(ctx, cudaMemcpyAsync(vcom_next, vcom_prev, size_t(n) * 4, cudaMemcpyDeviceToDevice, st));
  if (sync) RAK_TRY(ctx, cudaMemsetAsync(aff_next, 0, size_t(n), st));
  else if (aff_next != aff_prev) RAK_TRY(ctx, cudaMemcpyAsync(aff_next, aff_prev, size_t(n), cudaMemcpyDeviceToDevice, st));
  rak::LpaArgs a{};
  a.off = gr->off; a.tgt = gr->tgt; a.wt = gr->wt; a.n = n;
  a.order = gr->order; a.rg = gr->rg;
  a.chunk_hub = gr->chunk_hub; a.hub_first = gr->hub_first; a.hub_chunk = gr->ly.hub_chunk; a.nchunks = gr->nchunks;
  if (sync) {
    a.vcom0 = const_cast<uint32_t *>(vcom_prev); a.vcom1 = vcom_next;
    a.aff0 = const_cast<uint8_t *>(aff_prev); a.aff1 = aff_next;
  } else {
    a.vcom0 = vcom_next; a.vcom1 = nullptr; a.aff0 = aff_next; a.aff1 = nullptr;
  }
  a.hub_arrive = b.arrive.as<uint32_t>(); a.hub_claim = b.claim.as<uint32_t>(); a.hub_moved = b.moved.as<int32_t>();
  a.sk_keys = b.skk.as<uint32_t>(); a.sk_wts = b.skw.as<float>();
  a.stats = b.stats.as<unsigned long long>(); a.rs = b.rs.p;
  a.iters = 1; a.start_iter = iteration; a.tolerance = r.tol; a.pickless_step = r.pickless;
  a.check_on_pickless = r.check_on_pickless; a.rescan = r.rescan; a.mark_test = rak::mark_test_for(a.n, gr->m); a.gpu_rule = r.rule == 2; a.timeout_ns = r.timeout_ns; a.tie_until = r.tie_until; a.stage = r.stage; a.grid_cap = r.max_blocks;
  int grid = 0;
  RAK_TRY(ctx, rak::launch_lpa(a, r.slots, r.mode, gr->off64, st, &grid));
  unsigned long long s[rak::STATS_STRIDE] = {};
  rak::RunStateHost hs{};
  RAK_TRY(ctx, cudaMemcpyAsync(s, b.stats.p, sizeof(s), cudaMemcpyDeviceToHost, st));
  RAK_TRY(ctx, cudaMemcpyAsync(&hs, b.rs.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
  RAK_TRY(ctx, cudaStreamSynchronize(st));
  if (hs.error) { set_err(ctx, "device-side wait gave up (status %u)", hs.error); return rak_status(hs.error); }
  if (changed) *changed = s[0];
  return RAK_OK;
}

rak_status rak_modularity_f64(rak_ctx *ctx, const rak_csr *g, const uint32_t *membership, double *q) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !g || !membership || !q) return RAK_ERR_INVALID_ARGUMENT;
  RAK_CHECK(check_csr_shape(ctx, g));
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  if (g->location == RAK_DEVICE) {
    DevBuf bad;
    unsigned int hbad = 0;
    RAK_TRY(ctx, bad.alloc(4, nullptr));
    RAK_TRY(ctx, cudaMemsetAsync(bad.p, 0, 4, ctx->stream));
    RAK_TRY(ctx, rak::launch_validate(g->offsets, g->offset_bits == 64, g->targets, g->n, g->m, bad.as<unsigned int>(), ctx->stream));
    RAK_TRY(ctx, cudaMemcpyAsync(&hbad, bad.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
    RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (hbad) { set_err(ctx, "invalid CSR (device check)"); return RAK_ERR_INVALID_CSR; }
    return modularity_dev(ctx, g->offsets, g->offset_bits == 64, g->targets, g->weights, g->n, membership, nullptr, q);
  }
  if (rak_csr_validate_host(g) != RAK_OK) { set_err(ctx, "invalid CSR (host check)"); return RAK_ERR_INVALID_CSR; }
  const int64_t n = g->n, m = g->m;
  const size_t ob = size_t(n + 1) * (g->offset_bits == 64 ? 8 : 4);
  DevBuf off, tgt, wt, lab;
  RAK_TRY(ctx, off.alloc(ob, nullptr));
  RAK_TRY(ctx, tgt.alloc(size_t(std::max<int64_t>(m, 1)) * 4, nullptr));
  if (g->weights) RAK_TRY(ctx, wt.alloc(size_t(std::max<int64_t>(m, 1)) * 4, nullptr));
  RAK_TRY(ctx, lab.alloc(size_t(std::max<int64_t>(n, 1)) * 4, nullptr));
  RAK_TRY(ctx, cudaMemcpyAsync(off.p, g->offsets, ob, cudaMemcpyHostToDevice, ctx->stream));
  if (m > 0) RAK_TRY(ctx, cudaMemcpyAsync(tgt.p, g->targets, size_t(m) * 4, cudaMemcpyHostToDevice, ctx->stream));
  if (g->weights && m > 0) RAK_TRY(ctx, cudaMemcpyAsync(wt.p, g->weights, size_t(m) * 4, cudaMemcpyHostToDevice, ctx->stream));
  if (n > 0) RAK_TRY(ctx, cudaMemcpyAsync(lab.p, membership, size_t(n) * 4, cudaMemcpyHostToDevice, ctx->stream));
  return modularity_dev(ctx, off.p, g->offset_bits == 64, tgt.as<uint32_t>(), wt.as<float>(), n, lab.as<uint32_t>(), nullptr, q);
}

rak_status rak_gen_rmat_device(rak_ctx *ctx, int scale, double edge_factor, double a, double b, double c,
                               uint64_t seed, float w_lo, float w_hi, int32_t offset_bits, rak_csr *out) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !out || scale < 1 || scale > 31 || !(edge_factor > 0) || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 ||
      w_hi < w_lo || (offset_bits != 32 && offset_bits != 64))
    return RAK_ERR_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  const int64_t samples = int64_t(std::llround(double(int64_t(1) << scale) * edge_factor));
  const uint32_t tA = uint32_t(std::lround(a * 65536.0));
  const uint32_t tAB = uint32_t(std::lround((a + b) * 65536.0));
  const uint32_t tABC = uint32_t(std::lround((a + b + c) * 65536.0));
  const bool weighted = !(w_lo == 1.0f && w_hi == 1.0f);
  rak::GenDeviceOut g{};
  const cudaError_t e = rak::gen_rmat_device(scale, samples, seed, tA, tAB, tABC, weighted, w_lo, w_hi,
                                             offset_bits == 64, ctx->stream, &g);
  if (e == cudaErrorInvalidValue) {
    set_err(ctx, "more edges than 32-bit offsets can index");
    return RAK_ERR_INVALID_ARGUMENT;
  }
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    set_err(ctx, "device memory: the build needs about 16 bytes per sampled edge direction");
    return RAK_ERR_OUT_OF_MEMORY;
  }
  RAK_TRY(ctx, e);
  out->n = g.n;
  out->m = g.m;
  out->offset_bits = offset_bits;
  out->location = RAK_DEVICE;
  out->offsets = g.offsets;
  out->targets = g.targets;
  out->weights = g.weights;
  return RAK_OK;
}

rak_status rak_gen_sbm_device(rak_ctx *ctx, int64_t n, int64_t k, double avg_degree, double in_out_ratio, uint64_t seed,
                              int32_t offset_bits, rak_csr *out) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !out || n < 2 || n >= (int64_t(1) << 31) || k < 1 || k > n || !(avg_degree > 0) || !(in_out_ratio > 0) ||
      (offset_bits != 32 && offset_bits != 64))
    return RAK_ERR_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  // the host generator's parameters (rak_gen.cpp, rak_gen_sbm)
  const double s = double(n) / double(k);
  const double fin = k == 1 ? 1.0 : in_out_ratio * (s - 1) / (in_out_ratio * (s - 1) + (double(n) - s));
  const uint32_t fin24 = uint32_t(std::lround(fin * 16777216.0));
  const int64_t samples = int64_t(std::llround(double(n) * avg_degree / 2.0));
  rak::GenDeviceOut g{};
  const cudaError_t e = rak::gen_sbm_device(n, k, samples, fin24, seed, offset_bits == 64, ctx->stream, &g);
  if (e == cudaErrorInvalidValue) {
    set_err(ctx, "more edges than 32-bit offsets can index");
    return RAK_ERR_INVALID_ARGUMENT;
  }
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    set_err(ctx, "device memory: the build needs about 16 bytes per sampled edge direction");
    return RAK_ERR_OUT_OF_MEMORY;
  }
  RAK_TRY(ctx, e);
  out->n = g.n;
  out->m = g.m;
  out->offset_bits = offset_bits;
  out->location = RAK_DEVICE;
  out->offsets = g.offsets;
  out->targets = g.targets;
  out->weights = nullptr;
  return RAK_OK;
}

rak_status rak_device_csr_to_host(const rak_csr *g, rak_host_csr *out) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!g || !out || g->location != RAK_DEVICE || check_csr_shape(nullptr, g) != RAK_OK) return RAK_ERR_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  const int64_t n = g->n, m = g->m;
  out->offsets = static_cast<int64_t *>(std::malloc(size_t(n + 1) * 8));
  out->targets = static_cast<uint32_t *>(std::malloc(size_t(std::max<int64_t>(m, 1)) * 4));
  if (g->weights) out->weights = static_cast<float *>(std::malloc(size_t(std::max<int64_t>(m, 1)) * 4));
  if (!out->offsets || !out->targets || (g->weights && !out->weights)) {
    rak_host_csr_free(out);
    return RAK_ERR_OUT_OF_MEMORY;
  }
  cudaError_t e = cudaSuccess;
  if (g->offset_bits == 64) {
    e = cudaMemcpy(out->offsets, g->offsets, size_t(n + 1) * 8, cudaMemcpyDeviceToHost);
  } else {
    std::vector<int32_t> o32(size_t(n + 1));
    e = cudaMemcpy(o32.data(), g->offsets, size_t(n + 1) * 4, cudaMemcpyDeviceToHost);
    for (int64_t u = 0; u <= n; ++u) out->offsets[u] = o32[size_t(u)];
  }
  if (e == cudaSuccess && m > 0) e = cudaMemcpy(out->targets, g->targets, size_t(m) * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && m > 0 && g->weights) e = cudaMemcpy(out->weights, g->weights, size_t(m) * 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    rak_host_csr_free(out);
    return RAK_ERR_CUDA;
  }
  out->n = n;
  out->m = m;
  return RAK_OK;
}

rak_status rak_reference_vertex_order(rak_ctx *ctx, const rak_csr *g, uint32_t *ks) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !g || !ks || g->location != RAK_DEVICE) return RAK_ERR_INVALID_ARGUMENT;
  RAK_CHECK(check_csr_shape(ctx, g));
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  if (g->n == 0) return RAK_OK;
  DevBuf pos, scratch;
  RAK_TRY(ctx, pos.alloc(size_t(g->n) * 4, nullptr));
  RAK_TRY(ctx, scratch.alloc(rak::ref_order_scratch_bytes(g->n, 1), nullptr));
  RAK_TRY(ctx, rak::ref_order(g->offsets, g->offset_bits == 64, g->n, nullptr, nullptr, 0, ks, pos.as<uint32_t>(),
                              scratch.p, ctx->stream));
  RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return RAK_OK;
}

rak_status rak_batch_reference_vertex_order(rak_ctx *ctx, rak_batch *b, uint32_t *ks) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !b || !b->g || !ks) return RAK_ERR_INVALID_ARGUMENT;
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  const int64_t n = b->g->n, G = b->ngraphs;
  if (n == 0) return RAK_OK;
  DevBuf order, pos, scratch;
  RAK_TRY(ctx, order.alloc(size_t(n) * 4, nullptr));
  RAK_TRY(ctx, pos.alloc(size_t(n) * 4, nullptr));
  RAK_TRY(ctx, scratch.alloc(rak::ref_order_scratch_bytes(n, G), nullptr));
  RAK_TRY(ctx, rak::ref_order(b->g->off, true, n, b->gid.as<uint32_t>(), b->vbase.as<int64_t>(), G,
                              order.as<uint32_t>(), pos.as<uint32_t>(), scratch.p, ctx->stream));
  // global vertex indices to graph-local ids
  RAK_TRY(ctx, rak::launch_batch_finish(order.as<uint32_t>(), nullptr, nullptr, b->gid.as<uint32_t>(),
                                        b->vbase.as<int64_t>(), n, ks, ctx->stream));
  RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return RAK_OK;
}

rak_status rak_device_csr_free(rak_csr *g) {
  if (!g || g->location != RAK_DEVICE) return RAK_ERR_INVALID_ARGUMENT;
  cudaFree(const_cast<void *>(g->offsets));
  cudaFree(const_cast<uint32_t *>(g->targets));
  cudaFree(const_cast<float *>(g->weights));
  std::memset(g, 0, sizeof(*g));
  return RAK_OK;
}

rak_status rak_csr_validate_host(const rak_csr *g) {
  if (check_csr_shape(nullptr, g) != RAK_OK) return RAK_ERR_INVALID_ARGUMENT;
  if (g->location != RAK_HOST) return RAK_ERR_INVALID_ARGUMENT;
  if (g->offset_bits == 64)
    return validate_host_t(static_cast<const int64_t *>(g->offsets), g->targets, g->n, g->m);
  return validate_host_t(static_cast<const int32_t *>(g->offsets), g->targets, g->n, g->m);
}

rak_status rak_plan_summary_host(const rak_csr *g, const rak_options *o, int64_t counts[8], int64_t *hub_chunks) {
  if (!g || !counts || check_csr_shape(nullptr, g) != RAK_OK || g->location != RAK_HOST) return RAK_ERR_INVALID_ARGUMENT;
  Resolved r;
  rak_status s = resolve(nullptr, o, &r);
  if (s != RAK_OK) return s;
  for (int i = 0; i < 8; ++i) counts[i] = 0;
  int64_t ch = 0;
  for (int64_t u = 0; u < g->n; ++u) {
    const int64_t deg = g->offset_bits == 64
        ? static_cast<const int64_t *>(g->offsets)[u + 1] - static_cast<const int64_t *>(g->offsets)[u]
        : int64_t(static_cast<const int32_t *>(g->offsets)[u + 1]) - static_cast<const int32_t *>(g->offsets)[u];
    const uint32_t k = rak::plan_key(deg, r.ly);
    if (deg <= 0) { counts[7]++; continue; }
    const int reg = rak::key_region(k);
    // counts: lane groups 1,2,4,8,16,32 then split vertices
    if (reg == rak::REG_LANE) counts[0]++;
    else if (reg == rak::REG_HUB) { counts[6]++; ch += (deg + r.ly.hub_chunk - 1) / r.ly.hub_chunk; }
    else counts[6 - reg]++;  // region 5 (G=2) -> 1, ..., region 1 (G=32) -> 5
  }
  if (hub_chunks) *hub_chunks = ch;
  return RAK_OK;
}

}  // extern "C"

// ---- batches of graphs ----------------------------------------------------------------------

namespace {

rak_status batch_prepare(rak_ctx *ctx, rak_batch *b, const Resolved &r) {
  rak_graph *gr = b->g;
  if (!same_layout(gr->ly, r.ly)) RAK_CHECK(build_plan(ctx, gr, r.ly, nullptr));
  if (r.iters > 0) RAK_TRY(ctx, rak::prepare_lpa(r.slots, r.mode, true, gr->wt == nullptr, true, r.stage));
  const int64_t n = gr->n, G = b->ngraphs;
  const bool sync = r.mode != RAK_MODE_ASYNC;
  const int iters = std::max(r.iters, 1);
  RunBufs &rb = gr->bufs;
  RAK_TRY(ctx, ensure(rb.aff0, size_t(n) + 16));
  if (sync) {
    RAK_TRY(ctx, ensure(rb.vcom1, size_t(n) * 4 + 16));
    RAK_TRY(ctx, ensure(rb.aff1, size_t(n) + 16));
  }
  const size_t nh = size_t(std::max<int64_t>(gr->nhub, 1)), nc = size_t(std::max<int64_t>(gr->nchunks, 1));
  RAK_TRY(ctx, ensure(rb.arrive, nh * 4));
  RAK_TRY(ctx, ensure(rb.claim, nh * 4));
  RAK_TRY(ctx, ensure(rb.moved, nh * 4));
  RAK_TRY(ctx, ensure(rb.skk, nc * size_t(r.slots) * 4));
  RAK_TRY(ctx, ensure(rb.skw, nc * size_t(r.slots) * 4));
  RAK_TRY(ctx, ensure(rb.stats, size_t(iters) * rak::STATS_STRIDE * 8));
  RAK_TRY(ctx, ensure(rb.rs, sizeof(rak::RunStateHost)));
  RAK_TRY(ctx, ensure(b->vcom0, size_t(n) * 4 + 16));
  RAK_TRY(ctx, ensure(b->gdone, size_t(G) + 16));
  RAK_TRY(ctx, ensure(b->giters, size_t(G) * 4 + 16));
  RAK_TRY(ctx, ensure(b->gchanged, size_t(G) * 16 + 16));
  RAK_TRY(ctx, ensure(b->running, size_t(iters) * 4 + 16));
  // asynchronous runs label by position in each graph's reference order (as a single graph does);
  // it depends on degrees only, so it is built once per packed batch
  if (r.order == 2 && n > 0 && !b->ref_ready) {
    RAK_TRY(ctx, ensure(b->ref_ks, size_t(n) * 4));
    RAK_TRY(ctx, ensure(b->ref_pos, size_t(n) * 4));
    RAK_TRY(ctx, ensure(b->ref_scratch, rak::ref_order_scratch_bytes(n, G)));
    RAK_TRY(ctx, rak::ref_order(gr->off, true, n, b->gid.as<uint32_t>(), b->vbase.as<int64_t>(), G,
                                b->ref_ks.as<uint32_t>(), b->ref_pos.as<uint32_t>(), b->ref_scratch.p, ctx->stream));
    if (!b->keep_ref_scratch) {
      RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
      b->ref_scratch.release();
    }
    b->ref_ready = true;
  }
  return RAK_OK;
}

// Enqueues the whole run; buffers must already be prepared (no allocation here, so the sequence
// is capturable).
rak_status batch_enqueue(rak_ctx *ctx, rak_batch *b, const uint32_t *q, const Resolved &r, uint32_t *membership,
                         int grid_cap = 0) {
  rak_graph *gr = b->g;
  RunBufs &rb = gr->bufs;
  cudaStream_t st = ctx->stream;
  const int64_t n = gr->n, G = b->ngraphs;
  const bool sync = r.mode != RAK_MODE_ASYNC;
  const int iters = std::max(r.iters, 1);
  RAK_TRY(ctx, cudaMemsetAsync(rb.arrive.p, 0, rb.arrive.bytes, st));
  RAK_TRY(ctx, cudaMemsetAsync(rb.claim.p, 0, rb.claim.bytes, st));
  RAK_TRY(ctx, cudaMemsetAsync(rb.moved.p, 0xFF, rb.moved.bytes, st));
  RAK_TRY(ctx, cudaMemsetAsync(rb.stats.p, 0, size_t(iters) * rak::STATS_STRIDE * 8, st));
  RAK_TRY(ctx, cudaMemsetAsync(rb.rs.p, 0, sizeof(rak::RunStateHost), st));
  RAK_TRY(ctx, cudaMemsetAsync(b->gdone.p, 0, size_t(G) + 16, st));
  RAK_TRY(ctx, cudaMemsetAsync(b->giters.p, 0, size_t(G) * 4 + 16, st));
  RAK_TRY(ctx, cudaMemsetAsync(b->gchanged.p, 0, size_t(G) * 16 + 16, st));
  RAK_TRY(ctx, cudaMemsetAsync(b->running.p, 0, size_t(iters) * 4 + 16, st));
  uint32_t *v1 = sync ? rb.vcom1.as<uint32_t>() : nullptr;
  const bool ref_labels = r.order == 2 && n > 0;
  if (ref_labels)
    RAK_TRY(ctx, rak::launch_batch_init_mapped(b->vcom0.as<uint32_t>(), q, b->gid.as<uint32_t>(), b->vbase.as<int64_t>(),
                                               b->ref_pos.as<uint32_t>(), n, st));
  else
    RAK_TRY(ctx, rak::launch_batch_init(b->vcom0.as<uint32_t>(), v1, q, b->gid.as<uint32_t>(), b->vbase.as<int64_t>(), n, st));
  RAK_TRY(ctx, rak::launch_init_flags(rb.aff0.as<uint8_t>(), sync ? rb.aff1.as<uint8_t>() : nullptr, nullptr, n, st));
  if (r.iters > 0) {
    rak::LpaArgs a{};
    a.off = gr->off; a.tgt = gr->tgt; a.wt = gr->wt; a.n = n;
    a.order = gr->order; a.rg = gr->rg;
    a.chunk_hub = gr->chunk_hub; a.hub_first = gr->hub_first; a.hub_chunk = gr->ly.hub_chunk; a.nchunks = gr->nchunks;
    a.vcom0 = b->vcom0.as<uint32_t>(); a.vcom1 = v1; a.aff0 = rb.aff0.as<uint8_t>(); a.aff1 = sync ? rb.aff1.as<uint8_t>() : nullptr;
    a.hub_arrive = rb.arrive.as<uint32_t>(); a.hub_claim = rb.claim.as<uint32_t>(); a.hub_moved = rb.moved.as<int32_t>();
    a.sk_keys = rb.skk.as<uint32_t>(); a.sk_wts = rb.skw.as<float>();
    a.stats = rb.stats.as<unsigned long long>(); a.rs = rb.rs.p;
    a.gid = b->gid.as<uint32_t>(); a.vbase = b->vbase.as<int64_t>(); a.gdone = b->gdone.as<uint8_t>();
    a.giters = b->giters.as<int32_t>(); a.gchanged = b->gchanged.as<unsigned long long>();
    a.running = b->running.as<unsigned int>(); a.ngraphs = G; a.grid_cap = grid_cap > 0 ? grid_cap : r.max_blocks;
    a.iters = r.iters; a.start_iter = r.start; a.tolerance = r.tol; a.pickless_step = r.pickless;
    a.check_on_pickless = r.check_on_pickless; a.rescan = r.rescan; a.mark_test = rak::mark_test_for_batch(a.n, gr->m, G); a.gpu_rule = r.rule == 2; a.timeout_ns = r.timeout_ns; a.tie_until = r.tie_until; a.stage = r.stage;
    int grid = 0;
    RAK_TRY(ctx, rak::launch_lpa(a, r.slots, r.mode, true, st, &grid, true));
  }
  if (ref_labels)
    RAK_TRY(ctx, rak::launch_batch_finish_mapped(b->vcom0.as<uint32_t>(), b->ref_ks.as<uint32_t>(), b->gid.as<uint32_t>(),
                                                 b->vbase.as<int64_t>(), n, membership, st));
  else
    RAK_TRY(ctx, rak::launch_batch_finish(b->vcom0.as<uint32_t>(), r.iters > 0 ? v1 : nullptr, rb.rs.p,
                                          b->gid.as<uint32_t>(), b->vbase.as<int64_t>(), n, membership, st));
  b->last_iters = iters;
  b->last_sync = sync;
  return RAK_OK;
}

}  // namespace

extern "C" {

rak_status rak_batch_create(rak_ctx *ctx, const rak_batch_csr *bc, const rak_options *o, rak_batch **out) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !bc || !out) return RAK_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (bc->graphs < 0 || !bc->graph_offsets) { set_err(ctx, "bad graph count or offsets"); return RAK_ERR_INVALID_ARGUMENT; }
  Resolved r;
  RAK_CHECK(resolve(ctx, o, &r));
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  rak_csr c{};
  c.n = bc->n; c.m = bc->m; c.offset_bits = 64; c.location = bc->location;
  c.offsets = bc->offsets; c.targets = bc->targets; c.weights = bc->weights;
  Resolved rn = r;
  rn.validate = 0;  // the batch rules (local target ids) are checked below
  if (r.validate && bc->location == RAK_HOST) {
    const int64_t *go = bc->graph_offsets, *off = bc->offsets;
    if (check_csr_shape(ctx, &c) != RAK_OK) return RAK_ERR_INVALID_ARGUMENT;
    bool ok = go[0] == 0 && go[bc->graphs] == bc->n && off[0] == 0 && off[bc->n] == bc->m;
    for (int64_t gi = 0; ok && gi < bc->graphs; ++gi) {
      if (go[gi] > go[gi + 1]) { ok = false; break; }
      const int64_t ng = go[gi + 1] - go[gi];
      for (int64_t u = go[gi]; ok && u < go[gi + 1]; ++u) {
        if (off[u] > off[u + 1]) ok = false;
        for (int64_t e = off[u]; ok && e < off[u + 1]; ++e) ok = int64_t(bc->targets[e]) < ng;
      }
    }
    if (!ok) { set_err(ctx, "invalid batch CSR (host check)"); return RAK_ERR_INVALID_CSR; }
  }
  auto *b = new (std::nothrow) rak_batch();
  if (!b) return RAK_ERR_OUT_OF_MEMORY;
  b->ctx = ctx;
  b->device = ctx->device;
  b->ngraphs = bc->graphs;
  struct Fail { rak_batch *b; bool armed = true; ~Fail() { if (armed) rak_batch_destroy(b); } } fail{b};
  RAK_CHECK(graph_create(ctx, &c, rn, nullptr, &b->g));
  const size_t gbytes = size_t(bc->graphs + 1) * 8;
  RAK_TRY(ctx, b->vbase.alloc(gbytes, nullptr));
  RAK_TRY(ctx, cudaMemcpyAsync(b->vbase.p, bc->graph_offsets, gbytes,
                               bc->location == RAK_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, ctx->stream));
  RAK_TRY(ctx, b->gid.alloc(size_t(std::max<int64_t>(bc->n, 1)) * 4, nullptr));
  RAK_TRY(ctx, rak::launch_batch_gid(b->vbase.as<int64_t>(), bc->graphs, bc->n, b->gid.as<uint32_t>(), ctx->stream));
  if (r.validate && bc->location == RAK_DEVICE) {
    DevBuf bad;
    unsigned int hbad = 0;
    RAK_TRY(ctx, bad.alloc(4, nullptr));
    RAK_TRY(ctx, cudaMemsetAsync(bad.p, 0, 4, ctx->stream));
    RAK_TRY(ctx, rak::launch_batch_validate(b->vbase.as<int64_t>(), bc->graphs, bc->n, static_cast<const int64_t *>(b->g->off),
                                            b->g->tgt, b->gid.as<uint32_t>(), bad.as<unsigned int>(), ctx->stream));
    RAK_TRY(ctx, cudaMemcpyAsync(&hbad, bad.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
    RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (hbad) { set_err(ctx, "invalid batch CSR (device check)"); return RAK_ERR_INVALID_CSR; }
  }
  RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  fail.armed = false;
  *out = b;
  return RAK_OK;
}

rak_status rak_batch_destroy(rak_batch *b) {
  if (!b) return RAK_ERR_INVALID_ARGUMENT;
  cudaSetDevice(b->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->g) rak_graph_destroy(b->g);
  delete b;
  return RAK_OK;
}

rak_status rak_batch_launch(rak_ctx *ctx, rak_batch *b, const uint32_t *q, const rak_options *o, uint32_t *membership) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !b || !membership) return RAK_ERR_INVALID_ARGUMENT;
  Resolved r;
  RAK_CHECK(resolve(ctx, o, &r));
  batch_default_order(o, &r);
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  RAK_CHECK(batch_prepare(ctx, b, r));
  return batch_enqueue(ctx, b, q, r, membership);
}

rak_status rak_batch_results(rak_ctx *ctx, rak_batch *b, int32_t *iterations, rak_result *total) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !b) return RAK_ERR_INVALID_ARGUMENT;
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  RunBufs &rb = b->g->bufs;
  rak::RunStateHost hs{};
  if (!rb.rs.p) { set_err(ctx, "no launch yet"); return RAK_ERR_INVALID_ARGUMENT; }
  RAK_TRY(ctx, cudaMemcpy(&hs, rb.rs.p, sizeof(hs), cudaMemcpyDeviceToHost));
  if (hs.error) { set_err(ctx, "device-side wait gave up (status %u)", hs.error); return rak_status(hs.error); }
  if (iterations && b->ngraphs > 0)
    RAK_TRY(ctx, cudaMemcpy(iterations, b->giters.p, size_t(b->ngraphs) * 4, cudaMemcpyDeviceToHost));
  if (total) {
    std::memset(total, 0, sizeof(*total));
    total->modularity = std::numeric_limits<double>::quiet_NaN();
    std::vector<unsigned long long> st(size_t(b->last_iters) * rak::STATS_STRIDE);
    RAK_TRY(ctx, cudaMemcpy(st.data(), rb.stats.p, st.size() * 8, cudaMemcpyDeviceToHost));
    const int done = int(std::min<unsigned>(hs.iterations, unsigned(b->last_iters)));
    total->iterations = done;
    for (int i = 0; i < done; ++i) {
      const unsigned long long *x = &st[size_t(i) * rak::STATS_STRIDE];
      total->traversed_edges += x[rak::STAT_EDGES];
      total->processed_vertices += x[rak::STAT_PROCESSED];
      total->moved_vertices += x[rak::STAT_CHANGED];
      total->moved_edges += x[rak::STAT_MOVED_EDGES];
      total->marked_edges += x[rak::STAT_MOVED_EDGES];   // batches mark after every move
    }
    total->changed_last = done > 0 ? st[size_t(done - 1) * rak::STATS_STRIDE + rak::STAT_CHANGED] : 0;
    total->plan_ms = b->g->plan_ms;
    const uint64_t bytes = b->g->graph_bytes + b->g->plan_bytes + rb.bytes() + b->vbase.bytes + b->gid.bytes +
                           b->vcom0.bytes + b->gdone.bytes + b->giters.bytes + b->gchanged.bytes + b->running.bytes +
                           b->ref_ks.bytes + b->ref_pos.bytes + b->ref_scratch.bytes;
    total->peak_device_bytes = bytes;
    total->memory_gb = float(double(bytes - b->g->graph_bytes) / (1024.0 * 1024.0 * 1024.0));
  }
  return RAK_OK;
}

rak_status rak_batch_capture(rak_ctx *ctx, rak_batch *b, const uint32_t *q, const rak_options *o, uint32_t *membership) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !b || !membership) return RAK_ERR_INVALID_ARGUMENT;
  Resolved r;
  RAK_CHECK(resolve(ctx, o, &r));
  batch_default_order(o, &r);
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  RAK_CHECK(batch_prepare(ctx, b, r));  // allocations happen before the capture
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
  RAK_TRY(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  rak_status s = batch_enqueue(ctx, b, q, r, membership);
  cudaGraph_t gph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(ctx->stream, &gph);
  if (s != RAK_OK) { if (gph) cudaGraphDestroy(gph); return s; }
  RAK_TRY(ctx, e);
  b->graph = gph;
  RAK_TRY(ctx, cudaGraphInstantiate(&b->exec, gph, 0));
  return RAK_OK;
}

rak_status rak_batch_replay(rak_ctx *ctx, rak_batch *b) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !b || !b->exec) return RAK_ERR_INVALID_ARGUMENT;
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  RAK_TRY(ctx, cudaGraphLaunch(b->exec, ctx->stream));
  return RAK_OK;
}

rak_status rak_batch_modularity_f64(rak_ctx *ctx, rak_batch *b, const uint32_t *membership, double *q) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !b || !membership || !q) return RAK_ERR_INVALID_ARGUMENT;
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  const int64_t n = b->g->n, G = b->ngraphs;
  DevBuf ctot, gs;
  RAK_TRY(ctx, ctot.alloc(size_t(std::max<int64_t>(n, 1)) * 8, nullptr));
  RAK_TRY(ctx, gs.alloc(size_t(3 * G + 1) * 8, nullptr));
  RAK_TRY(ctx, cudaMemsetAsync(ctot.p, 0, ctot.bytes, ctx->stream));
  RAK_TRY(ctx, cudaMemsetAsync(gs.p, 0, gs.bytes, ctx->stream));
  double *gin = gs.as<double>(), *gtot = gin + G, *gsq = gtot + G, *bad = gsq + G;
  if (n > 0)
    RAK_TRY(ctx, rak::launch_batch_modularity(static_cast<const int64_t *>(b->g->off), b->g->tgt, b->g->wt,
                                              b->gid.as<uint32_t>(), b->vbase.as<int64_t>(), n, membership,
                                              ctot.as<double>(), gin, gtot, gsq, bad, ctx->stream));
  std::vector<double> h(size_t(3 * G + 1));
  RAK_TRY(ctx, cudaMemcpyAsync(h.data(), gs.p, h.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
  RAK_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (h[size_t(3 * G)] > 0) { set_err(ctx, "membership holds labels beyond their graph"); return RAK_ERR_INVALID_ARGUMENT; }
  for (int64_t gi = 0; gi < G; ++gi) {
    const double in = h[size_t(gi)], tot = h[size_t(G + gi)], sq = h[size_t(2 * G + gi)];
    q[gi] = tot > 0 ? in / tot - sq / (tot * tot) : 0.0;
  }
  return RAK_OK;
}

}  // extern "C"

// ---- serving: continuous batching -----------------------------------------------------------

namespace {

using Clock = std::chrono::steady_clock;

struct ServerRequest {
  uint64_t ticket = 0;
  rak_csr g{};        // the caller's arrays, host or device (valid until completion)
  uint64_t bytes = 0; // budget held while admitted
  Clock::time_point t_submit, t_launch, t_done;
  std::vector<uint32_t> membership;
  int32_t iterations = 0;
  rak_status status = RAK_OK;
  bool done = false;
};
using ReqPtr = std::shared_ptr<ServerRequest>;

// Page-locked host buffer, grown only when too small.
struct Pinned {
  void *p = nullptr;
  size_t bytes = 0;
  Pinned() = default;
  Pinned(const Pinned &) = delete;
  Pinned &operator=(const Pinned &) = delete;
  ~Pinned() { if (p) cudaFreeHost(p); }
  cudaError_t ensure(size_t b) {
    if (p && bytes >= b) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    const size_t want = std::max<size_t>(b + b / 2 + 4096, size_t(1) << 20);
    cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
    if (e == cudaSuccess) bytes = want;
    else p = nullptr;
    return e;
  }
  template <class T> T *as() const { return static_cast<T *>(p); }
};

// One launch slot: its own context (stream), a reusable batch and staging buffers.
struct ServerSlot {
  rak_ctx *ctx = nullptr;
  rak_batch *b = nullptr;
  Pinned h_go, h_mem, h_it, h_bad;
  DevBuf d_mem, d_items, d_bad, d_stage;
  cudaMemPool_t pool = nullptr;  // stream-ordered device allocations of this slot
  cudaEvent_t ev = nullptr;
  std::vector<ReqPtr> reqs;
  std::vector<int64_t> vo;
  Clock::time_point t_launch;
  bool busy = false;       // holds requests
  bool launching = false;  // requests taken, event not recorded yet
};

// Budget charged for a request: its graph plus per-vertex labels, flags and plan.
uint64_t request_bytes(const rak_csr &g) {
  const uint64_t n = uint64_t(g.n), m = uint64_t(g.m);
  return 8 * (n + 1) + 4 * m + (g.weights ? 4 * m : 0) + 32 * n + 256;
}

// Grows an owned device array of a slot's batch graph (contents are not kept), stream-ordered
// from the slot's pool (the caller holds a PoolScope).
cudaError_t grow(rak_graph *gr, const void *&p, size_t &cap, size_t need) {
  if (p && cap >= need) return cudaSuccess;
  rak_host_detail::dev_free(const_cast<void *>(p), gr->arrays_pooled, gr->arrays_fs);
  p = nullptr;
  cap = 0;
  void *q = nullptr;
  const size_t want = need + need / 2 + 256;
  cudaError_t e = rak_host_detail::dev_alloc(&q, want, &gr->arrays_fs);
  if (e != cudaSuccess) return e;
  gr->arrays_pooled = rak_host_detail::thread_pool().pool != nullptr;
  p = q;
  cap = want;
  return cudaSuccess;
}

}  // namespace

struct rak_server {
  rak_ctx *ctx = nullptr;
  int device = 0;
  rak_server_options opt{};
  Resolved run{};
  int grid_cap = 0;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<ReqPtr> pending;
  std::unordered_map<uint64_t, ReqPtr> tickets;
  std::vector<std::unique_ptr<ServerSlot>> slots;
  uint64_t used = 0, next_ticket = 1;
  bool stop = false;
  rak_server_stats st{};
};

namespace {

// Fails the slot's requests whose flag in bad[] is set (graphs that break the CSR rules) and
// drops them from the slot.
void server_drop_invalid(rak_server *s, ServerSlot &sl, const unsigned int *bad) {
  std::vector<ReqPtr> keep;
  std::lock_guard<std::mutex> lk(s->mu);
  const auto now = Clock::now();
  for (size_t i = 0; i < sl.reqs.size(); ++i) {
    if (!bad[i]) { keep.push_back(sl.reqs[i]); continue; }
    ServerRequest &r = *sl.reqs[i];
    r.status = RAK_ERR_INVALID_CSR;
    r.done = true;
    r.t_done = now;
    s->used -= r.bytes;
    s->st.rejected++;
  }
  sl.reqs = std::move(keep);
  s->cv_done.notify_all();
}

// Packs the slot's requests into its batch on the device. Host-located graphs: targets and
// weights uploaded straight into their place, offsets uploaded as they are into a staging area.
// One gather kernel then rebases every graph's offsets and copies the edges of device-located
// graphs, checking the CSR rules; with validation on, the flags are read back and failing graphs
// are dropped before the plan is built (host graphs were checked at submission).
rak_status server_load(rak_server *s, ServerSlot &sl) {
  rak_ctx *ctx = sl.ctx;
  cudaStream_t st = ctx->stream;
  const auto t0 = Clock::now();
  for (;;) {
    const size_t G = sl.reqs.size();
    if (G == 0) return RAK_OK;
    sl.vo.assign(G + 1, 0);
    std::vector<int64_t> eo(G + 1, 0), so(G + 1, 0);  // first edge slot; staging byte offset
    int64_t max_elems = 0;
    bool weighted = false;
    for (size_t i = 0; i < G; ++i) {
      const rak_csr &g = sl.reqs[i]->g;
      sl.vo[i + 1] = sl.vo[i] + g.n;
      eo[i + 1] = eo[i] + g.m;
      const int64_t ob = g.location == RAK_HOST ? ((g.n + 1) * (g.offset_bits / 8) + 15) / 16 * 16 : 0;
      so[i + 1] = so[i] + ob;
      weighted |= g.weights != nullptr;
      max_elems = std::max(max_elems, std::max(g.n, g.location == RAK_DEVICE ? g.m : 0));
    }
    const int64_t n_tot = sl.vo[G], m_tot = eo[G];
    if (!sl.b) {
      auto *b = new (std::nothrow) rak_batch();
      auto *gr = new (std::nothrow) rak_graph();
      if (!b || !gr) { delete b; delete gr; return RAK_ERR_OUT_OF_MEMORY; }
      gr->ctx = ctx;
      gr->device = ctx->device;
      gr->owns = true;
      gr->off64 = true;
      b->ctx = ctx;
      b->device = ctx->device;
      b->g = gr;
      b->keep_ref_scratch = true;
      sl.b = b;
    }
    rak_batch *b = sl.b;
    rak_graph *gr = b->g;
    RAK_TRY(ctx, grow(gr, gr->off, gr->off_cap, size_t(n_tot + 1) * 8));
    const void *tp = gr->tgt;
    RAK_TRY(ctx, grow(gr, tp, gr->tgt_cap, size_t(std::max<int64_t>(m_tot, 1)) * 4));
    gr->tgt = static_cast<const uint32_t *>(tp);
    if (weighted) {
      const void *wp = gr->wt_alloc;
      RAK_TRY(ctx, grow(gr, wp, gr->wt_cap, size_t(std::max<int64_t>(m_tot, 1)) * 4));
      gr->wt_alloc = const_cast<void *>(wp);
    }
    gr->n = n_tot;
    gr->m = m_tot;
    gr->wt = weighted ? static_cast<const float *>(gr->wt_alloc) : nullptr;
    gr->graph_bytes = gr->off_cap + gr->tgt_cap + gr->wt_cap;
    int64_t *d_off = static_cast<int64_t *>(const_cast<void *>(gr->off));
    uint32_t *d_tgt = const_cast<uint32_t *>(gr->tgt);
    float *d_wt = weighted ? static_cast<float *>(gr->wt_alloc) : nullptr;
    RAK_TRY(ctx, ensure(sl.d_stage, size_t(std::max<int64_t>(so[G], 16))));
    char *stage = sl.d_stage.as<char>();
    // pinned: graph vertex offsets (G + 1), the final edge offset, then the gather items
    RAK_TRY(ctx, sl.h_go.ensure((G + 2) * 8 + G * sizeof(rak::GatherItem) + 64));
    int64_t *go = sl.h_go.as<int64_t>();
    auto *items = reinterpret_cast<rak::GatherItem *>(go + G + 2);
    for (size_t i = 0; i <= G; ++i) go[i] = sl.vo[i];
    go[G + 1] = m_tot;
    for (size_t i = 0; i < G; ++i) {
      const rak_csr &g = sl.reqs[i]->g;
      rak::GatherItem &it = items[i];
      it.n = g.n;
      it.m = g.m;
      it.vdst = sl.vo[i];
      it.edst = eo[i];
      it.off64 = g.offset_bits == 64;
      it.pad = 0;
      if (g.location == RAK_DEVICE) {
        it.off = g.offsets;
        it.tgt = g.targets;
        it.wt = g.weights;
        continue;
      }
      it.off = stage + so[i];
      it.tgt = nullptr;
      it.wt = nullptr;
      RAK_TRY(ctx, cudaMemcpyAsync(stage + so[i], g.offsets, size_t(g.n + 1) * (g.offset_bits / 8),
                                   cudaMemcpyHostToDevice, st));
      if (g.m > 0) {
        RAK_TRY(ctx, cudaMemcpyAsync(d_tgt + eo[i], g.targets, size_t(g.m) * 4, cudaMemcpyHostToDevice, st));
        if (weighted && g.weights)
          RAK_TRY(ctx, cudaMemcpyAsync(d_wt + eo[i], g.weights, size_t(g.m) * 4, cudaMemcpyHostToDevice, st));
        else if (weighted) RAK_TRY(ctx, rak::launch_fill_f32(d_wt + eo[i], g.m, 1.0f, st));
      }
    }
    RAK_TRY(ctx, ensure(sl.d_items, G * sizeof(rak::GatherItem)));
    RAK_TRY(ctx, ensure(sl.d_bad, G * 4));
    RAK_TRY(ctx, cudaMemcpyAsync(sl.d_items.p, items, G * sizeof(rak::GatherItem), cudaMemcpyHostToDevice, st));
    RAK_TRY(ctx, cudaMemcpyAsync(d_off + n_tot, go + G + 1, 8, cudaMemcpyHostToDevice, st));
    RAK_TRY(ctx, cudaMemsetAsync(sl.d_bad.p, 0, G * 4, st));
    RAK_TRY(ctx, rak::launch_gather_graphs(sl.d_items.as<rak::GatherItem>(), int(G), max_elems, d_off, d_tgt, d_wt,
                                           sl.d_bad.as<unsigned int>(), st));
    if (s->run.validate) {
      RAK_TRY(ctx, sl.h_bad.ensure(G * 4));
      RAK_TRY(ctx, cudaMemcpyAsync(sl.h_bad.p, sl.d_bad.p, G * 4, cudaMemcpyDeviceToHost, st));
      RAK_TRY(ctx, cudaStreamSynchronize(st));
      const unsigned int *bad = sl.h_bad.as<unsigned int>();
      bool any = false;
      for (size_t i = 0; i < G; ++i) any |= bad[i] != 0;
      if (any) {
        server_drop_invalid(s, sl, bad);
        continue;  // pack the remaining requests again
      }
    }
    b->ngraphs = int64_t(G);
    RAK_TRY(ctx, ensure(b->vbase, (G + 1) * 8));
    RAK_TRY(ctx, cudaMemcpyAsync(b->vbase.p, go, (G + 1) * 8, cudaMemcpyHostToDevice, st));
    RAK_TRY(ctx, ensure(b->gid, size_t(std::max<int64_t>(n_tot, 1)) * 4));
    RAK_TRY(ctx, rak::launch_batch_gid(b->vbase.as<int64_t>(), int64_t(G), n_tot, b->gid.as<uint32_t>(), st));
    b->ref_ready = false;  // a new set of graphs: its reference order is built by batch_prepare
    const auto t1 = Clock::now();
    const rak_status ps = build_plan(ctx, gr, s->run.ly, nullptr);
    const auto t2 = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.pack_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
    s->st.plan_host_ms += std::chrono::duration<double, std::milli>(t2 - t1).count();
    return ps;
  }
}

rak_status server_launch(rak_server *s, ServerSlot &sl) {
  rak_host_detail::PoolScope scope(sl.pool, sl.ctx->stream);
  const auto t0 = Clock::now();
  RAK_CHECK(server_load(s, sl));
  if (sl.reqs.empty()) return RAK_OK;  // every request failed its check
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.load_ms += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    s->st.plan_ms += sl.b->g->plan_ms;
  }
  sl.t_launch = Clock::now();
  rak_ctx *ctx = sl.ctx;
  rak_batch *b = sl.b;
  const int64_t n = b->g->n, G = b->ngraphs;
  RAK_CHECK(batch_prepare(ctx, b, s->run));
  RAK_TRY(ctx, ensure(sl.d_mem, size_t(std::max<int64_t>(n, 1)) * 4));
  const auto t_prepared = Clock::now();
  RAK_TRY(ctx, sl.h_mem.ensure(size_t(std::max<int64_t>(n, 1)) * 4));
  RAK_TRY(ctx, sl.h_it.ensure(size_t(std::max<int64_t>(G, 1)) * 4));
  RAK_CHECK(batch_enqueue(ctx, b, nullptr, s->run, sl.d_mem.as<uint32_t>(), s->grid_cap));
  RAK_TRY(ctx, cudaMemcpyAsync(sl.h_mem.p, sl.d_mem.p, size_t(n) * 4, cudaMemcpyDeviceToHost, ctx->stream));
  RAK_TRY(ctx, cudaMemcpyAsync(sl.h_it.p, b->giters.p, size_t(G) * 4, cudaMemcpyDeviceToHost, ctx->stream));
  RAK_TRY(ctx, cudaEventRecord(sl.ev, ctx->stream));
  std::lock_guard<std::mutex> lk(s->mu);
  s->st.enqueue_ms += std::chrono::duration<double, std::milli>(Clock::now() - t_prepared).count();
  return RAK_OK;
}

void server_loop(rak_server *s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    int inflight = 0;
    for (auto &slp : s->slots) {
      ServerSlot &sl = *slp;
      if (!sl.busy || sl.launching) { inflight += sl.busy; continue; }
      if (cudaEventQuery(sl.ev) != cudaSuccess) { ++inflight; continue; }
      const auto now = Clock::now();
      const uint32_t *mem = sl.h_mem.as<uint32_t>();
      const int32_t *its = sl.h_it.as<int32_t>();
      for (size_t i = 0; i < sl.reqs.size(); ++i) {
        ServerRequest &r = *sl.reqs[i];
        r.membership.assign(mem + sl.vo[i], mem + sl.vo[i + 1]);
        r.iterations = its[i];
        r.t_done = now;
        r.done = true;
        s->used -= r.bytes;
        s->st.completed++;
        s->st.edges_completed += uint64_t(r.g.m);
      }
      s->st.run_ms += std::chrono::duration<double, std::milli>(now - sl.t_launch).count();
      sl.reqs.clear();
      sl.busy = false;
      s->cv_done.notify_all();
    }
    ServerSlot *free_slot = nullptr;
    for (auto &slp : s->slots)
      if (!slp->busy) { free_slot = slp.get(); break; }
    if (free_slot && !s->pending.empty()) {
      std::vector<ReqPtr> sel;
      uint64_t bytes = 0;
      while (!s->pending.empty() && int(sel.size()) < s->opt.max_graphs_per_launch) {
        ReqPtr r = s->pending.front();
        if (r->bytes > s->opt.budget_bytes) {  // can never fit
          s->pending.pop_front();
          r->status = RAK_ERR_OUT_OF_MEMORY;
          r->done = true;
          r->t_done = Clock::now();
          s->st.rejected++;
          s->cv_done.notify_all();
          continue;
        }
        if (s->used + bytes + r->bytes > s->opt.budget_bytes) break;
        sel.push_back(r);
        bytes += r->bytes;
        s->pending.pop_front();
      }
      if (!sel.empty()) {
        s->used += bytes;
        const auto now = Clock::now();
        for (auto &r : sel) r->t_launch = now;
        free_slot->reqs = std::move(sel);
        free_slot->busy = true;
        free_slot->launching = true;
        s->st.launches++;
        s->st.graphs_launched += free_slot->reqs.size();
        s->st.max_concurrent_launches = std::max(s->st.max_concurrent_launches, inflight + 1);
        lk.unlock();
        const rak_status rs = server_launch(s, *free_slot);
        lk.lock();
        free_slot->launching = false;
        if (rs == RAK_OK && free_slot->reqs.empty()) free_slot->busy = false;
        if (rs != RAK_OK) {
          for (auto &r : free_slot->reqs) {
            r->status = rs;
            r->done = true;
            r->t_done = Clock::now();
            s->used -= r->bytes;
          }
          free_slot->reqs.clear();
          free_slot->busy = false;
          s->cv_done.notify_all();
        }
        continue;
      }
    }
    if (s->stop && s->pending.empty() && inflight == 0) break;
    s->cv_work.wait_for(lk, std::chrono::microseconds(inflight > 0 ? 50 : 1000));
  }
}

}  // namespace

extern "C" {

void rak_server_options_default(rak_server_options *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->budget_bytes = uint64_t(16) << 30;
  o->max_graphs_per_launch = 256;
  o->slots = 2;
  o->queue_capacity = 65536;
  rak_options_default(&o->run);
}

rak_status rak_server_create(rak_ctx *ctx, const rak_server_options *o, rak_server **out) {
  if (!ctx || !out) return RAK_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  rak_server_options d;
  rak_server_options_default(&d);
  if (!o) o = &d;
  if (o->slots < 1 || o->slots > 16 || o->max_graphs_per_launch < 1 || o->queue_capacity < 1) {
    set_err(ctx, "server options out of range");
    return RAK_ERR_INVALID_ARGUMENT;
  }
  auto *s = new (std::nothrow) rak_server();
  if (!s) return RAK_ERR_OUT_OF_MEMORY;
  s->ctx = ctx;
  s->device = ctx->device;
  s->opt = *o;
  rak_status st = resolve(ctx, &o->run, &s->run);
  batch_default_order(&o->run, &s->run);
  if (st != RAK_OK) { delete s; return st; }
  s->grid_cap = std::max(1, ctx->sms * 3 / o->slots);
  for (int i = 0; i < o->slots; ++i) {
    s->slots.push_back(std::make_unique<ServerSlot>());
    ServerSlot &sl = *s->slots.back();
    st = rak_ctx_create(ctx->device, &sl.ctx);
    if (st == RAK_OK && cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess) st = RAK_ERR_CUDA;
    if (st == RAK_OK) {
      // the slot's own pool keeps what it has allocated (release threshold: everything), so a
      // slot's buffers, once grown, are reused without going back to the driver
      cudaMemPoolProps props{};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = ctx->device;
      uint64_t keep = ~uint64_t(0);
      if (cudaMemPoolCreate(&sl.pool, &props) != cudaSuccess ||
          cudaMemPoolSetAttribute(sl.pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
        st = RAK_ERR_CUDA;
    }
    if (st != RAK_OK) {
      for (auto &x : s->slots) {
        if (x->pool) cudaMemPoolDestroy(x->pool);
        if (x->ev) cudaEventDestroy(x->ev);
        if (x->ctx) rak_ctx_destroy(x->ctx);
      }
      delete s;
      return st;
    }
  }
  s->worker = std::thread(server_loop, s);
  *out = s;
  return RAK_OK;
}

rak_status rak_server_submit(rak_server *s, const rak_csr *g, uint64_t *ticket) {
  if (!s || !g || !ticket) return RAK_ERR_INVALID_ARGUMENT;
  if (check_csr_shape(nullptr, g) != RAK_OK || (g->location != RAK_HOST && g->location != RAK_DEVICE))
    return RAK_ERR_INVALID_ARGUMENT;
  // host graphs are checked here, on the caller's thread; device graphs when their launch is packed
  if (g->location == RAK_HOST && s->run.validate && rak_csr_validate_host(g) != RAK_OK) return RAK_ERR_INVALID_CSR;
  auto r = std::make_shared<ServerRequest>();
  r->g = *g;
  r->bytes = request_bytes(*g);
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return RAK_ERR_INVALID_ARGUMENT;
    if (int64_t(s->pending.size()) >= s->opt.queue_capacity) return RAK_ERR_BUSY;
    r->ticket = s->next_ticket++;
    s->tickets[r->ticket] = r;
    s->pending.push_back(r);
    s->st.submitted++;
  }
  s->cv_work.notify_one();
  *ticket = r->ticket;
  return RAK_OK;
}

rak_status rak_server_wait(rak_server *s, uint64_t ticket, double timeout_s, uint32_t *membership, rak_result *res) {
  if (!s) return RAK_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return RAK_ERR_INVALID_ARGUMENT;
  ReqPtr r = it->second;
  const auto limit = std::chrono::duration<double>(timeout_s < 0 ? 0.0 : timeout_s);
  if (!s->cv_done.wait_for(lk, limit, [&] { return r->done; })) return RAK_ERR_TIMEOUT;
  s->tickets.erase(it);
  lk.unlock();
  if (res) {
    std::memset(res, 0, sizeof(*res));
    res->modularity = std::numeric_limits<double>::quiet_NaN();
    res->iterations = r->iterations;
    res->time_ms = float(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
    const auto started = r->status == RAK_OK ? r->t_launch : r->t_done;
    res->plan_ms = float(std::chrono::duration<double, std::milli>(started - r->t_submit).count());
  }
  if (r->status != RAK_OK) return r->status;
  if (membership && !r->membership.empty()) std::memcpy(membership, r->membership.data(), r->membership.size() * 4);
  return RAK_OK;
}

rak_status rak_server_stats_get(rak_server *s, rak_server_stats *out) {
  if (!s || !out) return RAK_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->device_bytes_in_use = s->used;
  out->pending = int32_t(s->pending.size());
  return RAK_OK;
}

rak_status rak_server_destroy(rak_server *s) {
  if (!s) return RAK_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->device);
  for (auto &slp : s->slots) {
    ServerSlot &sl = *slp;
    if (sl.ctx) cudaStreamSynchronize(sl.ctx->stream);
    if (sl.b) rak_batch_destroy(sl.b);  // pooled buffers are freed on the slot's stream
    sl.b = nullptr;
    for (DevBuf *d : {&sl.d_mem, &sl.d_items, &sl.d_bad, &sl.d_stage}) d->release();
    if (sl.ctx) cudaStreamSynchronize(sl.ctx->stream);
    if (sl.pool) cudaMemPoolDestroy(sl.pool);
    if (sl.ev) cudaEventDestroy(sl.ev);
    if (sl.ctx) rak_ctx_destroy(sl.ctx);
  }
  delete s;
  return RAK_OK;
}

}  // extern "C"
