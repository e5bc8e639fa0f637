// rak_lowmem.hpp -- C++ drop-in for the reference's GPU label propagation entry points, over the
// C ABI of librak_lowmem.so (rak_lowmem.h). Header-only; link with -lrak_lowmem.
//
//   rak_b200::rakLowmemStaticCuda<SLOTS>(x, o)   <- rakLowmemStaticCuda<SLOTS>(x, o)
//                                                  (inc/rakLowmemCuda.hxx:624-632)
//   rak_b200::rakLowmemCuda(x, q, o, slots)       <- rakLowmemInvokeCuda(x, o, fi, fm) with fi
//                                                  initialising labels from q (:538-607)
//   rak_b200::RakOptions / RakResult<K>           <- RakOptions, RakResult<K> (inc/rak.hxx:19-97)
//
// G is any graph type with the reference's interface: key_type, span(), order(),
// forEachVertexKey(f(u)), forEachEdge(u, f(v, w)) (inc/Graph.hxx). As in the reference, the CSR is
// built on the host over the vertices that exist (in forEachVertexKey order) and membership has
// span() entries. Community names are vertex keys of x (the reference uses indices of its internal
// vertex order; both are arbitrary names). Errors throw rak_b200::Error with the rak_status
// instead of exiting the process (the reference's TRY_CUDA calls exit()).
#pragma once
#include <cstdint>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "rak_lowmem.h"

namespace rak_b200 {

struct RakOptions {
  int repeat;
  double tolerance;
  int maxIterations;
  RakOptions(int repeat = 1, double tolerance = 0.05, int maxIterations = 20)
      : repeat(repeat), tolerance(tolerance), maxIterations(maxIterations) {}
};

template <class K>
struct RakResult {
  std::vector<K> membership;
  int iterations = 0;
  float time = 0;                // ms
  float markingTime = 0;         // ms
  float initializationTime = 0;  // ms
  float memory = 0;              // GB of working buffers beyond the graph
  uint64_t traversedEdges = 0;   // sum over iterations of the degrees of processed vertices
  uint64_t peakDeviceBytes = 0;  // everything the run held on the device, graph included
  RakResult() = default;
  RakResult(std::vector<K> &&membership, int iterations = 0, float time = 0, float markingTime = 0,
            float initializationTime = 0, float memory = 0)
      : membership(std::move(membership)), iterations(iterations), time(time), markingTime(markingTime),
        initializationTime(initializationTime), memory(memory) {}
};

class Error : public std::runtime_error {
 public:
  rak_status status;
  Error(rak_status s, const std::string &what) : std::runtime_error(what), status(s) {}
};

inline void check(rak_status s, const rak_ctx *ctx = nullptr) {
  if (s == RAK_OK) return;
  std::string msg = rak_status_string(s);
  if (ctx && *rak_ctx_last_error(ctx)) msg += std::string(": ") + rak_ctx_last_error(ctx);
  throw Error(s, msg);
}

// One context per process for `device`, created on first use and kept until exit (the reference
// runs on the current device's default stream).
inline rak_ctx *defaultContext(int device = 0) {
  static std::mutex mu;
  static rak_ctx *ctx[64] = {};
  if (device < 0 || device >= 64) throw Error(RAK_ERR_INVALID_ARGUMENT, "device out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!ctx[device]) check(rak_ctx_create(device, &ctx[device]));
  return ctx[device];
}

// The host CSR of x over its existing vertices, in forEachVertexKey order (csr.hxx:126-297 with
// the identity key order).
template <class G>
struct HostCsr {
  using K = typename G::key_type;
  std::vector<K> keys;           // index -> vertex key
  std::vector<int64_t> offsets;
  std::vector<uint32_t> targets;
  std::vector<float> weights;
  explicit HostCsr(const G &x) {
    const size_t S = x.span();
    std::vector<uint32_t> index(S, 0);
    keys.reserve(x.order());
    x.forEachVertexKey([&](auto u) { index[size_t(u)] = uint32_t(keys.size()); keys.push_back(K(u)); });
    offsets.reserve(keys.size() + 1);
    offsets.push_back(0);
    for (K u : keys) {
      x.forEachEdge(u, [&](auto v, auto w) {
        targets.push_back(index[size_t(v)]);
        weights.push_back(float(w));
      });
      offsets.push_back(int64_t(targets.size()));
    }
  }
  rak_csr csr() const {
    rak_csr c{};
    c.n = int64_t(keys.size());
    c.m = int64_t(targets.size());
    c.offset_bits = 64;
    c.location = RAK_HOST;
    c.offsets = offsets.data();
    c.targets = targets.empty() ? nullptr : targets.data();
    c.weights = weights.empty() ? nullptr : weights.data();
    return c;
  }
};

// Label propagation with an optional initial membership q (indexed by vertex key, values are
// vertex keys; nullptr: every vertex starts in its own community). `extra` carries the options the
// reference fixes at compile time or not at all (mode, rescan, layout, ...); its repeat,
// tolerance, max_iterations and slots are taken from o and slots.
template <class G, class K = typename G::key_type>
RakResult<K> rakLowmemCuda(const G &x, const std::vector<K> *q, const RakOptions &o, int slots = 8,
                           const rak_options *extra = nullptr, int device = 0) {
  HostCsr<G> h(x);
  const size_t n = h.keys.size();
  rak_options opt;
  if (extra) opt = *extra;
  else rak_options_default(&opt);
  opt.repeat = o.repeat;
  opt.tolerance = o.tolerance;
  opt.max_iterations = o.maxIterations;
  opt.slots = slots;
  std::vector<uint32_t> q32, labels(n);
  if (q) {
    std::vector<uint32_t> index(x.span(), 0);
    for (size_t i = 0; i < n; ++i) index[size_t(h.keys[i])] = uint32_t(i);
    q32.resize(n);
    for (size_t i = 0; i < n; ++i) q32[i] = index[size_t((*q)[size_t(h.keys[i])])];
  }
  rak_ctx *ctx = defaultContext(device);
  rak_result r{};
  const rak_csr c = h.csr();
  check(rak_lowmem_cuda(ctx, &c, q ? q32.data() : nullptr, &opt, labels.data(), &r), ctx);
  std::vector<K> membership(x.span(), K());
  for (size_t i = 0; i < n; ++i) membership[size_t(h.keys[i])] = h.keys[labels[i]];
  RakResult<K> out(std::move(membership), r.iterations, r.time_ms, r.marking_time_ms, r.initialization_time_ms,
                   r.memory_gb);
  out.traversedEdges = r.traversed_edges;
  out.peakDeviceBytes = r.peak_device_bytes;
  return out;
}

// rakLowmemStaticCuda<SLOTS,RESCAN,TRYWARP,TRYMERGE>(x, o): SLOTS = 1 is νBM-LPA, 8 is νMG8-LPA.
// RESCAN, TRYWARP and TRYMERGE select implementation details of the reference's kernels; the
// asynchronous mode here has no rescan (the reference's default), so they are accepted and unused.
template <int SLOTS = 8, bool RESCAN = false, bool TRYWARP = true, bool TRYMERGE = true, class G>
inline auto rakLowmemStaticCuda(const G &x, const RakOptions &o = {}) {
  static_assert(SLOTS == 1 || SLOTS == 2 || SLOTS == 4 || SLOTS == 8 || SLOTS == 16, "SLOTS: 1, 2, 4, 8 or 16");
  using K = typename G::key_type;
  return rakLowmemCuda<G, K>(x, static_cast<const std::vector<K> *>(nullptr), o, SLOTS);
}

}  // namespace rak_b200
