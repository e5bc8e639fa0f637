// rak_internal.hpp -- declarations shared by the host orchestration (rak_host.cpp) and the CUDA
// translation units. No CUDA device code here; plain structs passed to kernels by value.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace rak {

// Work regions of the degree-bucket plan, in processing order. The plan's vertex list `order`
// holds region 0's vertices first, then region 1's, and so on.
//   region 0      : split vertices (degree > hub_min), one item per chunk of hub_chunk edges,
//                   32 lanes per chunk
//   regions 1..5  : lane groups of G = 32, 16, 8, 4, 2 lanes per vertex
//   region 6      : one lane per vertex (1 <= degree <= lane_max), degree descending
// Isolated vertices (degree 0) are in no region: they can never move.
constexpr int NREG = 7;
constexpr int REG_HUB = 0;
constexpr int REG_LANE = 6;
__host__ __device__ constexpr int region_group(int r) { return r == REG_LANE ? 1 : (r == REG_HUB ? 32 : (64 >> r)); }

// Work items of region r holding cnt vertices (nchunks: split-vertex chunks, region 0; lane_item:
// batches of 32 one-lane vertices per item, region 6).
__host__ __device__ inline int64_t region_items(int r, int64_t cnt, int64_t nchunks, int64_t lane_item) {
  if (r == REG_HUB) return nchunks;
  if (r == REG_LANE) return (cnt + 32 * lane_item - 1) / (32 * lane_item);
  return (cnt * region_group(r) + 31) / 32;
}
// Batches of 32 one-lane vertices per work item. Each item is claimed with one atomic on the
// launch-wide work counter: on low-degree graphs (tens of millions of one-lane vertices) items of
// 4 batches keep that counter from serialising the iteration (2D lattice 2^25: 1.06 -> 0.89 ms
// per iteration), while a graph with few one-lane vertices needs single batches to give every
// resident warp work (R-MAT scale 16: 2.5x slower with 4). warps: resident warps of a launch.
constexpr int LPA_WARPS_PER_SM = 32;  // lpa_run: 256-thread blocks, 4 resident per SM (RAK_MIN_BLOCKS)
inline int64_t lane_item_for(int64_t lane_vertices, int64_t warps) {
  const int64_t batches = (lane_vertices + 31) / 32, w = warps > 0 ? warps : 1;
  return batches >= 32 * w ? 4 : batches >= 16 * w ? 2 : 1;
}

struct Regions {
  int64_t vbegin[NREG];
  int64_t vcount[NREG];
  int64_t ibegin[NREG + 1];  // item prefix; ibegin[NREG] = total items
  int64_t lane_item;         // batches of 32 one-lane vertices per item (lane_item_for)
};

// Layout parameters (rak_options lane_max / hub_min / hub_chunk after defaults).
struct Layout {
  int64_t lane_max;
  int64_t hub_min;
  int64_t hub_chunk;
};
// Defaults chosen by the autotuner across R-MAT (scale 22-24, weighted and unit), planted SBM,
// lattice and batched-mix graphs: best or equal everywhere; on R-MAT the asynchronous iteration
// settles in 5-6 iterations instead of 20, since fewer vertices are split.
constexpr int64_t DEFAULT_LANE_MAX = 256;
constexpr int64_t DEFAULT_HUB_MIN = 65536;
constexpr int64_t DEFAULT_HUB_CHUNK = 8192;
constexpr int64_t MAX_LANE_MAX = 1024;
// Iterations with hashed ties (rak_options.tie_break 2) when rak_options.tie_iterations is 0.
constexpr int DEFAULT_TIE_ITERATIONS = 2;
// Edge staging (rak_options.edge_staging) when the option is 0: 1 on, 2 off.
constexpr int DEFAULT_EDGE_STAGING = 2;
// Dense iterations (rak_options.dense_pct) when the option is 0; a value <= 0 means never.
constexpr int DEFAULT_DENSE_PCT = -1;
// Bound on each device-side wait when rak_options.wait_timeout_ns is 0.
constexpr long long DEFAULT_WAIT_TIMEOUT_NS = 20LL * 1000 * 1000 * 1000;

// Sort key of a vertex in the plan (regions in order, region 6 by degree descending);
// key_isolated for degree 0. Shared by the device plan kernel and the host summary.
__host__ __device__ inline uint32_t plan_key(int64_t deg, const Layout &ly) {
  if (deg <= 0) return uint32_t(6 + ly.lane_max);
  if (deg <= ly.lane_max) return uint32_t(6 + (ly.lane_max - deg));
  if (deg > ly.hub_min) return 0u;
  int G = 2;
  while (G < 32 && int64_t(G) * ly.lane_max < deg) G *= 2;
  // G = 32 -> region 1, 16 -> 2, 8 -> 3, 4 -> 4, 2 -> 5
  int r = 1;
  for (int g = 32; g > G; g >>= 1) ++r;
  return uint32_t(r);
}
__host__ __device__ inline int key_region(uint32_t key) { return key < 6 ? int(key) : REG_LANE; }

struct RunStateHost {
  unsigned int bar, abort, error, iterations;
};

// Everything the persistent LPA kernel needs.
struct LpaArgs {
  const void *off;          // int32 or int64 offsets (template parameter of the kernel)
  const uint32_t *tgt;
  const float *wt;          // nullptr: unit weights
  int64_t n;
  const uint32_t *order;
  Regions rg;
  const uint32_t *chunk_hub;   // per chunk: index of its split vertex within region 0
  const int64_t *hub_first;    // per split vertex: first chunk (nhub+1 entries)
  int64_t hub_chunk;
  int64_t nchunks;
  uint32_t *vcom0, *vcom1;     // labels; vcom1 used by the synchronous modes
  uint8_t *aff0, *aff1;        // affected flags; aff1 used by the synchronous modes
  uint32_t *hub_arrive;        // per split vertex: chunks finished this iteration
  uint32_t *hub_claim;         // per split vertex: (iteration+1)<<1 | active, asynchronous mode
  int32_t *hub_moved;          // per split vertex: last iteration it moved in (-1: never)
  uint32_t *sk_keys;           // per chunk: slots keys of its partial sketch
  float *sk_wts;               // per chunk: slots weights
  unsigned long long *stats;   // per iteration, STATS_STRIDE slots (STAT_* below)
  void *rs;                    // RunState
  // Batches of independent graphs (BATCH kernels): targets are ids local to their graph.
  const uint32_t *gid;          // per vertex: index of its graph
  const int64_t *vbase;         // per graph: first vertex (ngraphs+1 entries)
  uint8_t *gdone;               // per graph: converged (its vertices are no longer processed)
  int32_t *giters;              // per graph: iterations it ran
  unsigned long long *gchanged; // 2*ngraphs: vertices changed per graph, this and next iteration
  unsigned int *running;        // per iteration: graphs still running after it
  int64_t ngraphs;
  int grid_cap;                 // at most this many blocks (0: as many as fit), to share the GPU
  int mark_test;                // neighbour marking reads a flag before storing it (mark_test_for)
  int gpu_rule;                 // synchronous split mode: the reference GPU sketch rules (else CPU)
  int tie_until;                // iterations l < tie_until break Misra-Gries ties by hash (CPU rules)
  int stage;                    // warp-wide edge ranges read through shared-memory tiles (bulk copies)
  int iters;
  int start_iter;
  double tolerance;
  int pickless_step;
  int check_on_pickless;
  int rescan;
  long long timeout_ns;
  // asynchronous single graphs: an iteration marks no neighbours (and the next processes every
  // vertex) when the previous iteration's moved vertices hold at least this many edges; 0: never
  unsigned long long dense_moved_edges;
};

enum Mode { MODE_ASYNC = 0, MODE_SYNC = 1, MODE_SPLIT = 2 };

// Edges that the moved vertices of an iteration must hold for the next iteration of an
// asynchronous single-graph run to mark no neighbours (LpaArgs::dense_moved_edges); 0: never.
inline unsigned long long dense_threshold(int mode, int pct_option, int64_t m) {
  const int pct = pct_option == 0 ? DEFAULT_DENSE_PCT : pct_option;
  if (mode != MODE_ASYNC || pct <= 0 || m <= 0) return 0ull;
  return (unsigned long long)((m * int64_t(pct) + 99) / 100);
}

// Label order (rak_options.label_order) of single-graph runs when the option is 0: vertex ids (1),
// except asynchronous runs with one or two slots, which take the reference GPU path's order (2).
// Measured on B200: a sketch too small to hold a degree-4 neighbourhood (Boyer-Moore, MG2) ends on
// the last neighbour it saw, on a grid-numbered graph the largest neighbour id, which the pickless
// first iteration forbids, and with id labels the run stalls (lattice, Boyer-Moore: Q 0.003
// against 0.607); larger Misra-Gries sketches hold the neighbourhood, break the tie by hash and are
// faster on R-MAT with id labels. Synchronous modes always label by id.
inline int default_label_order(int mode, int slots) { return mode == MODE_ASYNC && slots <= 2 ? 2 : 1; }

// Per-iteration counters written by the LPA kernel.
// STAT_PHASE: how the iteration treated the frontier (bit 0: its moves marked no neighbours; bit 1:
// it processed every vertex), written by the asynchronous single-graph kernel.
enum Stat { STAT_CHANGED = 0, STAT_EDGES = 1, STAT_PROCESSED = 2, STAT_HUBS_MOVED = 3, STAT_MOVED_EDGES = 4, STAT_WORK = 5,
            STAT_PHASE = 6 };
constexpr int STATS_STRIDE = 8;

// Persistent cooperative launch of all iterations; grid chosen from occupancy. `batch` selects the
// kernels for concatenated batches of graphs (64-bit offsets only).
cudaError_t launch_lpa(const LpaArgs &a, int slots, int mode, bool off64, cudaStream_t st, int *grid_out,
                       bool batch = false);
// Per-slot-count instantiations (rak_lpa_s*.cu).
template <int S>
cudaError_t launch_lpa_slots(const LpaArgs &a, int mode, bool off64, bool batch, cudaStream_t st, int *grid_out);
template <int S>
cudaError_t resolve_lpa_slots(int mode, bool off64, bool unit, bool batch, bool stage, const void **fn, int *per_sm);
// Whether neighbour marking reads each flag (through L1) before storing it. Measured on B200 with
// the read through L1, test on / off, νMG8 and νBM: R-MAT scale 24 ef 32 (16.8 M vertices) 31.3 /
// 36.9 ms and 23.1 / 32.2 ms; R-MAT scale 27 ef 16 (134 M) 128.0 / 135.6 ms and 125.6 / 139.5 ms --
// many moved vertices mark the same flags, and a flag line in L1 answers without a request to L2.
// On smaller or sparser graphs the read only lengthens each moved vertex's marking: SBM 2 M
// vertices (degree 16) 1.43 / 1.33 ms, R-MAT scale 18 0.89 / 0.81 ms, SBM 100 k 0.83 / 0.32 ms,
// 2D lattice 2^25 (degree ~4) 12.8 / 12.0 ms. Single graphs test from 2^22 vertices with average
// degree 8 or more.
inline int mark_test_for(int64_t n, int64_t m) { return n >= (int64_t(1) << 22) && m >= 8 * n ? 1 : 0; }
// Batches (each graph's flags a compact range, its neighbours inside it): the single-graph rule at
// the batch's mean graph size.
inline int mark_test_for_batch(int64_t n, int64_t m, int64_t graphs) {
  return graphs > 0 ? mark_test_for(n / graphs, m / graphs) : 0;
}
// Loads and resolves the kernel a run will launch (outside its timed region).
cudaError_t prepare_lpa(int slots, int mode, bool off64, bool unit, bool batch, bool stage);

// Plan and utility kernels (rak_kernels.cu).
cudaError_t launch_validate(const void *off, bool off64, const uint32_t *tgt, int64_t n, int64_t m,
                            unsigned int *bad, cudaStream_t st);
cudaError_t launch_plan_keys(const void *off, bool off64, int64_t n, Layout ly, uint32_t *keys,
                             uint32_t *vids, unsigned long long *hist, int nkeys, cudaStream_t st);
cudaError_t plan_sort(uint32_t *keys_in, uint32_t *keys_out, uint32_t *vals_in, uint32_t *vals_out,
                      int64_t n, int end_bit, void *temp, size_t *temp_bytes, cudaStream_t st);
cudaError_t launch_init(uint32_t *vcom0, uint32_t *vcom1, const uint32_t *q, int64_t n, cudaStream_t st);
cudaError_t launch_init_flags(uint8_t *aff0, uint8_t *aff1, const uint8_t *f, int64_t n, cudaStream_t st);
// The reference GPU path's vertex order (partition by degree < 4, then < 128): ks (order) and pos
// (its inverse), and the label mappings between positions in it and vertex ids.
// gid/vbase/ngraphs: the graphs of a batch (ks, pos in global vertex indices), or null/0 for one graph.
size_t ref_order_scratch_bytes(int64_t n, int64_t ngraphs);
cudaError_t ref_order(const void *off, bool off64, int64_t n, const uint32_t *gid, const int64_t *vbase,
                      int64_t ngraphs, uint32_t *ks, uint32_t *pos, void *scratch, cudaStream_t st);
cudaError_t launch_init_mapped(uint32_t *vcom0, const uint32_t *q, const uint32_t *pos, int64_t n, cudaStream_t st);
// rak_renumber.cu: a copy of a graph renumbered in its plan's work order (new vertex i = order[i]);
// inv: old -> new; noff (n+1 entries), ntgt (m), nwt (m, or null for unit weights); ident: 0..n-1;
// deg: n+1 entries of the offset type. temp null: *temp_bytes receives the scan's space.
cudaError_t renumber_graph(const void *off, bool off64, const uint32_t *tgt, const float *wt, const uint32_t *order,
                           int64_t n, int64_t split, uint32_t *inv, void *deg, void *noff, uint32_t *ntgt, float *nwt,
                           uint32_t *ident, void *temp, size_t *temp_bytes, cudaStream_t st);
// Labels (q[order[i]] or order[i], through pos when given: labels as positions in the reference
// order) and flags (flags[order[i]] or 1) of new vertex i.
cudaError_t launch_renumbered_init(const uint32_t *order, const uint32_t *q, const uint32_t *pos, const uint8_t *flags,
                                   int64_t n, uint32_t *lab, uint8_t *aff, cudaStream_t st);
// out[v] = lab[inv[v]]: a run's labels back in the numbering of the graph as given.
cudaError_t launch_renumbered_gather(const uint32_t *lab, const uint32_t *inv, int64_t n, uint32_t *out,
                                     cudaStream_t st);
cudaError_t launch_labels_to_ids(uint32_t *m, const uint32_t *ks, int64_t n, cudaStream_t st);
cudaError_t launch_hub_degrees(const void *off, bool off64, const uint32_t *order, int64_t nhub,
                               int64_t *deg, cudaStream_t st);
cudaError_t launch_modularity(const void *off, bool off64, const uint32_t *tgt, const float *wt,
                              int64_t n, const uint32_t *labels, double *ctot, double *sums,
                              cudaStream_t st);

// Batches of graphs (rak_kernels.cu).
cudaError_t launch_fill_f32(float *p, int64_t count, float v, cudaStream_t st);
// Symmetric R-MAT on the device (rak_gen_device.cu); arrays allocated with cudaMalloc.
struct GenDeviceOut {
  void *offsets;
  uint32_t *targets;
  float *weights;
  int64_t n, m;
  uint64_t peak_bytes;  // device bytes held at the peak of the build
};
cudaError_t gen_rmat_device(int scale, int64_t samples, uint64_t seed, uint32_t tA, uint32_t tAB, uint32_t tABC,
                            bool weighted, float w_lo, float w_hi, bool off64, cudaStream_t st, GenDeviceOut *out);
// Planted-partition SBM on the device (rak_gen_device.cu), the samples of rak_gen_sbm.
cudaError_t gen_sbm_device(int64_t n, int64_t k, int64_t samples, uint32_t fin24, uint64_t seed, bool off64,
                           cudaStream_t st, GenDeviceOut *out);
// One graph to pack into a batch CSR from device memory (k_gather_graphs).
struct GatherItem {
  const void *off;       // n + 1 offsets, int64 if off64 else int32
  const uint32_t *tgt;   // m targets (graph-local ids); null: edges already in place
  const float *wt;       // m weights, or null (unit)
  int64_t n, m;
  int64_t vdst, edst;    // first vertex and first edge slot in the batch
  int32_t off64, pad;
};
cudaError_t launch_gather_graphs(const GatherItem *items, int count, int64_t max_elems, int64_t *off_dst,
                                 uint32_t *tgt_dst, float *wt_dst, unsigned int *bad, cudaStream_t st);
cudaError_t launch_batch_gid(const int64_t *vbase, int64_t ngraphs, int64_t n, uint32_t *gid, cudaStream_t st);
cudaError_t launch_batch_validate(const int64_t *vbase, int64_t ngraphs, int64_t n, const int64_t *off,
                                  const uint32_t *tgt, const uint32_t *gid, unsigned int *bad, cudaStream_t st);
cudaError_t launch_batch_init(uint32_t *v0, uint32_t *v1, const uint32_t *q, const uint32_t *gid,
                              const int64_t *vbase, int64_t n, cudaStream_t st);
// Batch labels as global positions in each graph's reference order (q local), and back to local ids.
cudaError_t launch_batch_init_mapped(uint32_t *v0, const uint32_t *q, const uint32_t *gid, const int64_t *vbase,
                                     const uint32_t *pos, int64_t n, cudaStream_t st);
cudaError_t launch_batch_finish_mapped(const uint32_t *v0, const uint32_t *ks, const uint32_t *gid,
                                       const int64_t *vbase, int64_t n, uint32_t *membership, cudaStream_t st);
cudaError_t launch_batch_finish(const uint32_t *v0, const uint32_t *v1, const void *rs, const uint32_t *gid,
                                const int64_t *vbase, int64_t n, uint32_t *membership, cudaStream_t st);
cudaError_t launch_batch_modularity(const int64_t *off, const uint32_t *tgt, const float *wt, const uint32_t *gid,
                                    const int64_t *vbase, int64_t n, const uint32_t *labels, double *ctot,
                                    double *gin, double *gtot, double *gsq, double *bad, cudaStream_t st);

}  // namespace rak
