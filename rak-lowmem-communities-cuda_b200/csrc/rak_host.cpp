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
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "rak_internal.hpp"
#include "rak_lowmem.h"

struct rak_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own = nullptr;
  int sms = 0;
  std::string err;
};

namespace rak_host_detail {

// Device allocation that frees itself, with byte accounting for peak_device_bytes.
struct Tracker {
  uint64_t cur = 0, peak = 0;
  void add(uint64_t b) { cur += b; peak = std::max(peak, cur); }
  void sub(uint64_t b) { cur -= std::min(cur, b); }
};

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  Tracker *t = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) { cudaFree(p); if (t) t->sub(bytes); }
    p = nullptr;
    bytes = 0;
  }
  cudaError_t alloc(size_t b, Tracker *tr) {
    release();
    bytes = b ? b : 16;
    t = tr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) { p = nullptr; bytes = 0; return e; }
    if (t) t->add(bytes);
    return e;
  }
  template <class T> T *as() const { return static_cast<T *>(p); }
};

// Per-run device buffers, kept by a resident graph and reused while large enough.
struct RunBufs {
  DevBuf vcom1, aff0, aff1, arrive, claim, moved, skk, skw, stats, rs;
  uint64_t bytes() const {
    return vcom1.bytes + aff0.bytes + aff1.bytes + arrive.bytes + claim.bytes + moved.bytes + skk.bytes +
           skw.bytes + stats.bytes + rs.bytes;
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
  uint64_t graph_bytes = 0, plan_bytes = 0;
  float plan_ms = 0, h2d_ms = 0;
  rak_host_detail::RunBufs bufs;  // run buffers reused across runs
};

struct rak_batch {
  rak_ctx *ctx = nullptr;
  int device = 0;
  rak_graph *g = nullptr;           // the concatenated CSR (64-bit offsets) and its plan
  int64_t ngraphs = 0;
  rak_host_detail::DevBuf vbase, gid, vcom0, gdone, giters, gchanged, running;
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
cudaError_t ensure(DevBuf &d, size_t bytes) {
  if (d.p && d.bytes >= bytes) return cudaSuccess;
  return d.alloc(bytes, nullptr);
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
  int slots, mode, rescan, pickless, check_on_pickless, iters, start, validate, modularity, repeat;
  double tol;
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

rak_status check_csr_shape(rak_ctx *ctx, const rak_csr *g) {
  if (!g) { set_err(ctx, "null csr"); return RAK_ERR_INVALID_ARGUMENT; }
  if (g->n < 0 || g->n >= (int64_t(1) << 31) || g->m < 0) { set_err(ctx, "csr sizes out of range (n=%lld m=%lld)", (long long)g->n, (long long)g->m); return RAK_ERR_INVALID_ARGUMENT; }
  if (g->offset_bits != 32 && g->offset_bits != 64) { set_err(ctx, "offset_bits must be 32 or 64"); return RAK_ERR_INVALID_ARGUMENT; }
  if (g->offset_bits == 32 && g->m > int64_t(std::numeric_limits<int32_t>::max())) { set_err(ctx, "m too large for 32-bit offsets"); return RAK_ERR_INVALID_ARGUMENT; }
  if (g->location != RAK_HOST && g->location != RAK_DEVICE) { set_err(ctx, "bad location"); return RAK_ERR_INVALID_ARGUMENT; }
  if (!g->offsets || (g->m > 0 && !g->targets)) { set_err(ctx, "null csr arrays"); return RAK_ERR_INVALID_ARGUMENT; }
  return RAK_OK;
}

template <class O>
rak_status validate_host_t(const O *off, const uint32_t *tgt, int64_t n, int64_t m) {
  if (int64_t(off[0]) != 0 || int64_t(off[n]) != m) return RAK_ERR_INVALID_CSR;
  for (int64_t u = 0; u < n; ++u)
    if (off[u] > off[u + 1]) return RAK_ERR_INVALID_CSR;
  for (int64_t e = 0; e < m; ++e)
    if (int64_t(tgt[e]) >= n) return RAK_ERR_INVALID_CSR;
  return RAK_OK;
}

int nkeys_of(const Layout &ly) { return int(6 + ly.lane_max + 1); }

// Region sizes, item counts and chunk table from the key histogram and split-vertex degrees.
void regions_from(const std::vector<unsigned long long> &hist, const Layout &ly, int64_t nchunks, rak::Regions *rg) {
  int64_t cnt[rak::NREG] = {};
  for (int k = 0; k < 6; ++k) cnt[k] = int64_t(hist[k]);
  for (int64_t k = 6; k < 6 + ly.lane_max; ++k) cnt[rak::REG_LANE] += int64_t(hist[k]);
  int64_t v = 0, it = 0;
  for (int r = 0; r < rak::NREG; ++r) {
    rg->vbegin[r] = v;
    rg->vcount[r] = cnt[r];
    v += cnt[r];
    rg->ibegin[r] = it;
    const int G = rak::region_group(r);
    if (r == rak::REG_HUB) it += nchunks;
    else it += (cnt[r] * G + 31) / 32;
  }
  rg->ibegin[rak::NREG] = it;
}

rak_status build_plan(rak_ctx *ctx, rak_graph *gr, const Layout &ly, Tracker *tr) {
  cudaStream_t st = ctx->stream;
  cudaFree(gr->order); gr->order = nullptr;
  cudaFree(gr->chunk_hub); gr->chunk_hub = nullptr;
  cudaFree(gr->hub_first); gr->hub_first = nullptr;
  gr->plan_bytes = 0;
  gr->ly = ly;
  const int64_t n = gr->n;
  const int nk = nkeys_of(ly);
  Events ev;
  cudaEventRecord(ev.e[0], st);
  DevBuf keys, keys2, vids, hist, temp;
  RAK_TRY(ctx, keys.alloc(size_t(n) * 4, tr));
  RAK_TRY(ctx, keys2.alloc(size_t(n) * 4, tr));
  RAK_TRY(ctx, vids.alloc(size_t(n) * 4, tr));
  RAK_TRY(ctx, hist.alloc(size_t(nk) * 8, tr));
  RAK_TRY(ctx, cudaMalloc(&gr->order, size_t(std::max<int64_t>(n, 1)) * 4));
  gr->plan_bytes += size_t(std::max<int64_t>(n, 1)) * 4;
  if (tr) tr->add(size_t(std::max<int64_t>(n, 1)) * 4);
  RAK_TRY(ctx, cudaMemsetAsync(hist.p, 0, size_t(nk) * 8, st));
  std::vector<unsigned long long> h(size_t(nk), 0);
  if (n > 0) {
    RAK_TRY(ctx, rak::launch_plan_keys(gr->off, gr->off64, n, ly, keys.as<uint32_t>(), vids.as<uint32_t>(),
                                       hist.as<unsigned long long>(), nk, st));
    int end_bit = 1;
    while ((1 << end_bit) < nk) ++end_bit;
    size_t tb = 0;
    RAK_TRY(ctx, rak::plan_sort(keys.as<uint32_t>(), keys2.as<uint32_t>(), vids.as<uint32_t>(), gr->order, n,
                                end_bit, nullptr, &tb, st));
    RAK_TRY(ctx, temp.alloc(tb, tr));
    RAK_TRY(ctx, rak::plan_sort(keys.as<uint32_t>(), keys2.as<uint32_t>(), vids.as<uint32_t>(), gr->order, n,
                                end_bit, temp.p, &tb, st));
    RAK_TRY(ctx, cudaMemcpyAsync(h.data(), hist.p, size_t(nk) * 8, cudaMemcpyDeviceToHost, st));
    RAK_TRY(ctx, cudaStreamSynchronize(st));
  }
  gr->nhub = int64_t(h.empty() ? 0 : h[0]);
  gr->nchunks = 0;
  std::vector<int64_t> first(size_t(gr->nhub) + 1, 0);
  if (gr->nhub > 0) {
    DevBuf deg;
    RAK_TRY(ctx, deg.alloc(size_t(gr->nhub) * 8, tr));
    RAK_TRY(ctx, rak::launch_hub_degrees(gr->off, gr->off64, gr->order, gr->nhub, deg.as<int64_t>(), st));
    std::vector<int64_t> hd(size_t(gr->nhub));
    RAK_TRY(ctx, cudaMemcpyAsync(hd.data(), deg.p, size_t(gr->nhub) * 8, cudaMemcpyDeviceToHost, st));
    RAK_TRY(ctx, cudaStreamSynchronize(st));
    for (int64_t i = 0; i < gr->nhub; ++i) first[i + 1] = first[i] + (hd[i] + ly.hub_chunk - 1) / ly.hub_chunk;
    gr->nchunks = first[gr->nhub];
    std::vector<uint32_t> ch(size_t(gr->nchunks));
    for (int64_t i = 0; i < gr->nhub; ++i)
      for (int64_t c = first[i]; c < first[i + 1]; ++c) ch[c] = uint32_t(i);
    RAK_TRY(ctx, cudaMalloc(&gr->hub_first, first.size() * 8));
    RAK_TRY(ctx, cudaMalloc(&gr->chunk_hub, ch.size() * 4));
    gr->plan_bytes += first.size() * 8 + ch.size() * 4;
    if (tr) tr->add(first.size() * 8 + ch.size() * 4);
    RAK_TRY(ctx, cudaMemcpyAsync(gr->hub_first, first.data(), first.size() * 8, cudaMemcpyHostToDevice, st));
    RAK_TRY(ctx, cudaMemcpyAsync(gr->chunk_hub, ch.data(), ch.size() * 4, cudaMemcpyHostToDevice, st));
  }
  regions_from(h, ly, gr->nchunks, &gr->rg);
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
  } else {
    if (r.validate) {
      rak_status s = rak_csr_validate_host(g);
      if (s != RAK_OK) { set_err(ctx, "invalid CSR (host check)"); return fail(s); }
    }
    gr->owns = true;
    Events ev;
    void *po = nullptr, *pt = nullptr, *pw = nullptr;
    cudaError_t e = cudaMalloc(&po, ob);
    if (e == cudaSuccess) e = cudaMalloc(&pt, size_t(std::max<int64_t>(g->m, 1)) * 4);
    if (e == cudaSuccess && g->weights) e = cudaMalloc(&pw, size_t(std::max<int64_t>(g->m, 1)) * 4);
    gr->off = po; gr->tgt = static_cast<uint32_t *>(pt); gr->wt = static_cast<float *>(pw);
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
  if (g->location == RAK_DEVICE && r.validate) {
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
  a.check_on_pickless = r.check_on_pickless; a.rescan = r.rescan; a.timeout_ns = 20LL * 1000 * 1000 * 1000;

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
    RAK_TRY(ctx, rak::launch_init(vcom0, sync ? a.vcom1 : nullptr, q, n, st));
    cudaEventRecord(ev.e[1], st);
    RAK_TRY(ctx, rak::launch_init_flags(a.aff0, sync ? a.aff1 : nullptr, flags, n, st));
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
  if (sync && (done & 1)) RAK_TRY(ctx, cudaMemcpyAsync(vcom0, a.vcom1, size_t(n) * 4, cudaMemcpyDeviceToDevice, st));
  RAK_TRY(ctx, cudaStreamSynchronize(st));
  if (res) {
    res->iterations = done;
    res->time_ms = t_all / float(r.repeat);
    res->initialization_time_ms = t_init / float(r.repeat);
    res->marking_time_ms = t_mark / float(r.repeat);
    res->loop_ms = t_loop / float(r.repeat);
    res->traversed_edges = res->processed_vertices = res->moved_vertices = res->moved_edges = 0;
    for (int i = 0; i < done; ++i) {
      const unsigned long long *st_i = &stats[size_t(i) * rak::STATS_STRIDE];
      res->traversed_edges += st_i[rak::STAT_EDGES];
      res->processed_vertices += st_i[rak::STAT_PROCESSED];
      res->moved_vertices += st_i[rak::STAT_CHANGED];
      res->moved_edges += st_i[rak::STAT_MOVED_EDGES];
    }
    res->changed_last = done > 0 ? stats[size_t(done - 1) * rak::STATS_STRIDE + rak::STAT_CHANGED] : 0;
    res->memory_gb = float(double(b.bytes() + size_t(n) * 4 + gr->plan_bytes) / (1024.0 * 1024.0 * 1024.0));
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
  if (ctx->own) cudaStreamDestroy(ctx->own);
  delete ctx;
  return RAK_OK;
}

rak_status rak_ctx_set_stream(rak_ctx *ctx, void *stream) {
  if (!ctx) return RAK_ERR_INVALID_ARGUMENT;
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own;
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
    cudaFree(const_cast<void *>(gr->off));
    cudaFree(const_cast<uint32_t *>(gr->tgt));
    cudaFree(const_cast<float *>(gr->wt));
  }
  cudaFree(gr->order);
  cudaFree(gr->chunk_hub);
  cudaFree(gr->hub_first);
  delete gr;
  return RAK_OK;
}

uint64_t rak_graph_device_bytes(const rak_graph *gr) { return gr ? gr->graph_bytes + gr->plan_bytes : 0; }

rak_status rak_graph_run(rak_ctx *ctx, rak_graph *gr, const uint32_t *q, const rak_options *o,
                         uint32_t *membership, rak_result *res) {
  cudaGetLastError();  // drop a stale error left by an unrelated failed call
  if (!ctx || !gr || !membership) return RAK_ERR_INVALID_ARGUMENT;
  Resolved r;
  RAK_CHECK(resolve(ctx, o, &r));
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  Tracker tr;
  tr.add(gr->graph_bytes + gr->plan_bytes);
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
  RAK_TRY(ctx, cudaSetDevice(ctx->device));
  rak_result tmp{};
  rak_result *rr = res ? res : &tmp;
  std::memset(rr, 0, sizeof(*rr));
  rr->modularity = std::numeric_limits<double>::quiet_NaN();
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
  a.check_on_pickless = r.check_on_pickless; a.rescan = r.rescan; a.timeout_ns = 20LL * 1000 * 1000 * 1000;
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
  return RAK_OK;
}

// Enqueues the whole run; buffers must already be prepared (no allocation here, so the sequence
// is capturable).
rak_status batch_enqueue(rak_ctx *ctx, rak_batch *b, const uint32_t *q, const Resolved &r, uint32_t *membership) {
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
    a.running = b->running.as<unsigned int>(); a.ngraphs = G;
    a.iters = r.iters; a.start_iter = r.start; a.tolerance = r.tol; a.pickless_step = r.pickless;
    a.check_on_pickless = r.check_on_pickless; a.rescan = r.rescan; a.timeout_ns = 20LL * 1000 * 1000 * 1000;
    int grid = 0;
    RAK_TRY(ctx, rak::launch_lpa(a, r.slots, r.mode, true, st, &grid, true));
  }
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
  RAK_TRY(ctx, rak::launch_batch_gid(b->vbase.as<int64_t>(), bc->graphs, b->gid.as<uint32_t>(), ctx->stream));
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
    }
    total->changed_last = done > 0 ? st[size_t(done - 1) * rak::STATS_STRIDE + rak::STAT_CHANGED] : 0;
    total->plan_ms = b->g->plan_ms;
    const uint64_t bytes = b->g->graph_bytes + b->g->plan_bytes + rb.bytes() + b->vbase.bytes + b->gid.bytes +
                           b->vcom0.bytes + b->gdone.bytes + b->giters.bytes + b->gchanged.bytes + b->running.bytes;
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
