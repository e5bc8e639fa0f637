// rak_tune.cpp -- the autotuner: picks the degree thresholds (lane_max, hub_min), the split-vertex
// tile (hub_chunk) and the Misra-Gries slot count for a resident graph or a batch of graphs by
// running them. Written over the library's public C API only.
//
// Search: coordinate descent from the caller's options -- each dimension in turn (the label order
// of asynchronous runs, lane_max, hub_min, hub_chunk, slots) is swept with the others held at the
// best values so far, and the fastest candidate whose quality passes is kept. The label order
// goes first: it changes how fast the asynchronous iteration settles the most (R-MAT, whose hubs
// have small ids, settles sooner with id labels; under the reference's tie rule grid-numbered
// graphs stall with them and fail the quality gate). Objective: time to result (a run to convergence,
// best of `repeats`), since the layout also changes how fast the asynchronous iteration settles.
// Quality gate: FP64 modularity (mean over graphs for a batch) at least
// Q_start * (1 - quality_rel) - quality_abs, where Q_start is that of the caller's options.
// No reference counterpart (the reference fixes these at compile time).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <vector>

#include "rak_internal.hpp"
#include "rak_lowmem.h"

namespace {

struct Measured {
  rak_status st = RAK_OK;
  double ms = 0, q = 0, edges = 0;
  int iters = 0;
};

using Runner = std::function<Measured(const rak_options &)>;

bool layout_ok(const rak_options &o) {
  return o.lane_max >= 1 && o.lane_max <= 1024 && o.hub_min >= o.lane_max && o.hub_chunk >= 32 &&
         o.hub_chunk <= o.hub_min;
}

// single_graph: a run whose options leave the label order at 0 takes rak::default_label_order
// (by mode and slot count); batches label by vertex id.
rak_status search(const rak_tune_space *sp_in, const rak_options *base, bool single_graph, const Runner &run,
                  rak_options *best, rak_tune_entry *log, int32_t log_cap, int32_t *log_len) {
  rak_tune_space sp;
  if (sp_in) sp = *sp_in;
  else rak_tune_space_default(&sp);
  if (sp.n_lane_max < 0 || sp.n_lane_max > 8 || sp.n_hub_min < 0 || sp.n_hub_min > 8 || sp.n_hub_chunk < 0 ||
      sp.n_hub_chunk > 8 || sp.n_slots < 0 || sp.n_slots > 5 || sp.repeats < 1 || sp.label_orders < 0 ||
      sp.label_orders > 1)
    return RAK_ERR_INVALID_ARGUMENT;
  rak_options cur;
  if (base) cur = *base;
  else rak_options_default(&cur);
  cur.compute_modularity = 0;
  // zero means the library default: start from the values it stands for
  if (cur.lane_max == 0) cur.lane_max = int32_t(rak::DEFAULT_LANE_MAX);
  if (cur.hub_min == 0) cur.hub_min = int32_t(rak::DEFAULT_HUB_MIN);
  if (cur.hub_chunk == 0) cur.hub_chunk = int32_t(rak::DEFAULT_HUB_CHUNK);
  if (cur.label_order <= 0) cur.label_order = single_graph ? rak::default_label_order(cur.mode, cur.slots) : 1;
  int32_t n_log = 0;
  auto record = [&](const rak_options &o, const Measured &m, bool accepted) {
    if (log && n_log < log_cap) {
      rak_tune_entry &e = log[n_log];
      std::memset(&e, 0, sizeof(e));
      e.lane_max = o.lane_max;
      e.hub_min = o.hub_min;
      e.hub_chunk = o.hub_chunk;
      e.slots = o.slots;
      e.label_order = o.label_order;
      e.iterations = m.iters;
      e.accepted = accepted ? 1 : 0;
      e.ms = m.ms;
      e.modularity = m.q;
      e.edges_per_s = m.ms > 0 ? m.edges / (m.ms * 1e-3) : 0;
    }
    ++n_log;
  };
  const Measured first = run(cur);
  if (first.st != RAK_OK) return first.st;
  record(cur, first, true);
  const double q_floor = first.q * (1.0 - sp.quality_rel) - sp.quality_abs;
  double best_ms = first.ms;
  // one dimension at a time
  auto sweep = [&](int32_t rak_options::*field, const int32_t *vals, int32_t nv) -> rak_status {
    rak_options keep = cur;
    for (int32_t i = 0; i < nv; ++i) {
      rak_options o = cur;
      o.*field = vals[i];
      if (o.*field == cur.*field || !layout_ok(o)) continue;
      const Measured m = run(o);
      if (m.st == RAK_ERR_INVALID_ARGUMENT || m.st == RAK_ERR_UNSUPPORTED) continue;
      if (m.st != RAK_OK) return m.st;
      const bool pass = m.q >= q_floor;
      record(o, m, pass);
      if (pass && m.ms < best_ms) {
        best_ms = m.ms;
        keep = o;
      }
    }
    cur = keep;
    return RAK_OK;
  };
  rak_status s;
  const int32_t orders[] = {1, 2};
  if (sp.label_orders && cur.mode == RAK_MODE_ASYNC &&
      (s = sweep(&rak_options::label_order, orders, 2)) != RAK_OK)
    return s;
  if ((s = sweep(&rak_options::lane_max, sp.lane_max, sp.n_lane_max)) != RAK_OK) return s;
  if ((s = sweep(&rak_options::hub_min, sp.hub_min, sp.n_hub_min)) != RAK_OK) return s;
  if ((s = sweep(&rak_options::hub_chunk, sp.hub_chunk, sp.n_hub_chunk)) != RAK_OK) return s;
  if ((s = sweep(&rak_options::slots, sp.slots, sp.n_slots)) != RAK_OK) return s;
  if (best) {
    *best = cur;
    if (base) best->compute_modularity = base->compute_modularity;
  }
  if (log_len) *log_len = n_log;
  return RAK_OK;
}

}  // namespace

extern "C" {

void rak_tune_space_default(rak_tune_space *sp) {
  if (!sp) return;
  std::memset(sp, 0, sizeof(*sp));
  const int32_t lm[] = {32, 64, 128, 256};
  const int32_t hm[] = {4096, 8192, 16384, 32768, 65536};
  const int32_t hc[] = {2048, 4096, 8192, 16384};
  const int32_t sl[] = {4, 8, 16};
  std::copy(std::begin(lm), std::end(lm), sp->lane_max);
  sp->n_lane_max = 4;
  std::copy(std::begin(hm), std::end(hm), sp->hub_min);
  sp->n_hub_min = 5;
  std::copy(std::begin(hc), std::end(hc), sp->hub_chunk);
  sp->n_hub_chunk = 4;
  std::copy(std::begin(sl), std::end(sl), sp->slots);
  sp->n_slots = 3;
  sp->repeats = 2;
  sp->label_orders = 1;
  sp->quality_rel = 0.005;
  sp->quality_abs = 0.001;
}

rak_status rak_graph_autotune(rak_ctx *ctx, rak_graph *gr, const rak_options *base, const rak_tune_space *space,
                              uint32_t *membership, rak_options *best, rak_tune_entry *log, int32_t log_cap,
                              int32_t *log_len) {
  if (!ctx || !gr || !membership || log_cap < 0) return RAK_ERR_INVALID_ARGUMENT;
  const int repeats = space ? space->repeats : 2;
  Runner run = [&](const rak_options &o) {
    Measured m;
    rak_result r;
    m.st = rak_graph_run(ctx, gr, nullptr, &o, membership, &r);  // warm-up (and plan, if the layout changed)
    if (m.st != RAK_OK) return m;
    m.ms = std::numeric_limits<double>::infinity();
    for (int i = 0; i < std::max(1, repeats); ++i) {
      rak_options oq = o;
      oq.compute_modularity = i == 0;
      m.st = rak_graph_run(ctx, gr, nullptr, &oq, membership, &r);
      if (m.st != RAK_OK) return m;
      if (i == 0) m.q = r.modularity;
      if (r.time_ms < m.ms) {
        m.ms = r.time_ms;
        m.iters = r.iterations;
        m.edges = double(r.traversed_edges);
      }
    }
    return m;
  };
  return search(space, base, true, run, best, log, log_cap, log_len);
}

rak_status rak_batch_autotune(rak_ctx *ctx, rak_batch *b, int64_t graphs, const rak_options *base,
                              const rak_tune_space *space, uint32_t *membership, rak_options *best,
                              rak_tune_entry *log, int32_t log_cap, int32_t *log_len) {
  if (!ctx || !b || graphs < 0 || !membership || log_cap < 0) return RAK_ERR_INVALID_ARGUMENT;
  const int repeats = space ? space->repeats : 2;
  std::vector<double> q(size_t(std::max<int64_t>(graphs, 1)));
  Runner run = [&](const rak_options &o) {
    Measured m;
    rak_result r;
    m.st = rak_batch_launch(ctx, b, nullptr, &o, membership);  // warm-up (and plan, if the layout changed)
    if (m.st == RAK_OK) m.st = rak_batch_results(ctx, b, nullptr, &r);
    if (m.st != RAK_OK) return m;
    m.ms = std::numeric_limits<double>::infinity();
    for (int i = 0; i < std::max(1, repeats); ++i) {
      const auto t0 = std::chrono::steady_clock::now();
      m.st = rak_batch_launch(ctx, b, nullptr, &o, membership);
      if (m.st == RAK_OK) m.st = rak_batch_results(ctx, b, nullptr, &r);
      if (m.st != RAK_OK) return m;
      const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      if (ms < m.ms) {
        m.ms = ms;
        m.iters = r.iterations;
        m.edges = double(r.traversed_edges);
      }
    }
    m.st = rak_batch_modularity_f64(ctx, b, membership, q.data());
    if (m.st != RAK_OK) return m;
    double sum = 0;
    for (int64_t g = 0; g < graphs; ++g) sum += q[size_t(g)];
    m.q = graphs > 0 ? sum / double(graphs) : 0;
    return m;
  };
  return search(space, base, false, run, best, log, log_cap, log_len);
}

}  // extern "C"
