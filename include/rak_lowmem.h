/*
 * rak_lowmem.h -- C ABI of the B200-native memory-efficient label propagation library
 * (librak_lowmem.so): νMG-LPA (weighted Misra-Gries sketch, 2..16 slots; νMG8 = 8 slots) and
 * νBM-LPA (weighted Boyer-Moore vote) community detection on one GPU.
 *
 * The reference exposes its path as C++ templates; each entry point below names the reference
 * interface it replaces (paths relative to the reference repository):
 *   rak_lowmem_cuda        <- rakLowmemStaticCuda<SLOTS>(x, o)        inc/rakLowmemCuda.hxx:624-632
 *                             rakLowmemInvokeCuda(x, o, fi, fm)       inc/rakLowmemCuda.hxx:538-607
 *   rak_graph_create/run   <- the setup half (partition + CSR upload, :562-583) and the timed
 *                             loop half (:586-595) of rakLowmemInvokeCuda, split so a graph can
 *                             stay resident on the device across calls
 *   rak_graph_step         <- one move iteration, rakLowmemLoopCuU body  inc/rakLowmemCuda.hxx:476-487
 *   rak_modularity_f64     <- modularityBy(x, fc, M, R=1)            inc/properties.hxx:177-192
 *   rak_options            <- RakOptions{repeat,tolerance,maxIterations} inc/rak.hxx:19-40
 *   rak_result             <- RakResult<K>{membership,iterations,time,markingTime,
 *                             initializationTime,memory}             inc/rak.hxx:53-97
 *
 * Conventions. Every call returns a rak_status and never exits the process (the reference
 * prints and calls exit(), inc/_cuda.hxx:221-235). Vertex ids and labels are 0-based uint32.
 * Membership labels are vertex ids of the original graph (the reference returns indices into its
 * degree-partitioned order, inc/rakLowmemCuda.hxx:597-598; both are arbitrary community names).
 * A context is bound to one device and one stream and is not thread-safe; use one per thread.
 */
#ifndef RAK_LOWMEM_H
#define RAK_LOWMEM_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RAK_ABI_VERSION 1

typedef enum rak_status {
  RAK_OK = 0,
  RAK_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad option value, size out of range */
  RAK_ERR_INVALID_CSR = 2,      /* offsets not monotone / not ending at m, target id >= n */
  RAK_ERR_OUT_OF_MEMORY = 3,    /* device or host allocation failed, or admission budget exceeded */
  RAK_ERR_CUDA = 4,             /* a CUDA runtime call failed; see rak_ctx_last_error */
  RAK_ERR_TIMEOUT = 5,          /* a bounded device-side wait gave up */
  RAK_ERR_NO_DEVICE = 6,        /* no CUDA device, or the device is not sm_100 */
  RAK_ERR_UNSUPPORTED = 7,      /* option combination not implemented */
  RAK_ERR_BUSY = 8              /* serving: request queue full */
} rak_status;

typedef enum rak_location { RAK_HOST = 0, RAK_DEVICE = 1 } rak_location;

typedef enum rak_mode {
  /* In-place (Gauss-Seidel) label and flag updates, as the reference GPU path does
   * (inc/rakLowmemCuda.hxx:153,311,413). Split per-vertex sketches for high-degree vertices.
   * Defaults follow the reference GPU loop: pickless every 8th iteration, tolerance test
   * skipped on pickless iterations, no rescan. Nondeterministic, like the reference. */
  RAK_MODE_ASYNC = 0,
  /* Synchronous (Jacobi) iterations from a label snapshot, with every vertex scanned exactly in
   * edge order: bit-identical, iteration by iteration, to the reference's CPU per-vertex
   * functions (inc/rakLowmem.hxx:63-172) run on the same snapshot. Defaults follow the reference
   * CPU loop: rescan on, no pickless, tolerance tested every iteration. */
  RAK_MODE_SYNC = 1,
  /* Synchronous iterations with the split per-vertex sketches of RAK_MODE_ASYNC: deterministic,
   * and bit-identical to the documented split layout (rak_options.lane_max/hub_min/hub_chunk). */
  RAK_MODE_SYNC_SPLIT = 2
} rak_mode;

/* A graph in CSR form. All three arrays live in `location`. The graph should be symmetric
 * (undirected, both directions stored) as the reference's driver makes it (main.cxx:119). */
typedef struct rak_csr {
  int64_t n;              /* vertices, < 2^31 */
  int64_t m;              /* directed edges, == offsets[n] */
  int32_t offset_bits;    /* 32 or 64: element type of offsets */
  int32_t location;       /* rak_location */
  const void *offsets;    /* n+1 entries, offsets[0] == 0 */
  const uint32_t *targets;/* m entries, each < n */
  const float *weights;   /* m entries, or NULL for unit weights */
} rak_csr;

typedef struct rak_options {
  int32_t repeat;             /* RakOptions::repeat: runs averaged into time_ms [1] */
  double tolerance;           /* RakOptions::tolerance: stop when changed/n <= tolerance [0.05] */
  int32_t max_iterations;     /* RakOptions::maxIterations [20], <= 1024 */
  int32_t slots;              /* 1: νBM-LPA; 2, 4, 8, 16: νMG-LPA with that many slots [8] */
  int32_t mode;               /* rak_mode [RAK_MODE_ASYNC] */
  int32_t rescan;             /* -1: mode default; 1: exact weights of sketch keys (SYNC only) */
  int32_t pickless_step;      /* -1: mode default; 0: never; k: iterations l%k==0 only move to
                                 smaller labels (inc/rakLowmemCuda.hxx:473-476) */
  int32_t check_on_pickless;  /* -1: mode default; 1: tolerance tested on pickless iterations */
  int32_t lane_max;           /* 0: default [256]; split layout, one lane per vertex up to this degree */
  int32_t hub_min;            /* 0: default [65536]; vertices above this degree are split into chunks */
  int32_t hub_chunk;          /* 0: default [8192]; edges per chunk of a split vertex */
  int32_t validate;           /* 1: check the CSR on the device first [1] */
  int32_t compute_modularity; /* 1: fill rak_result.modularity (FP64 kernel) [0] */
  int32_t start_iteration;    /* iteration index of the first step (pickless schedule) [0] */
  const uint8_t *initial_flags; /* NULL: every vertex affected; else n flags in the csr's location */
  int32_t sketch_rule;        /* -1 or 0: mode default; 1: the reference CPU sketch rules (last free
                                 slot, clamped decrement, linear argmax, move if w > 0); 2: its GPU
                                 rules (first free slot, unclamped, tournament argmax, move if
                                 w != 0, Boyer-Moore from the own label). SYNC runs 1 only;
                                 ASYNC and SYNC_SPLIT run either [1] */
  int32_t label_order;        /* -1 or 0: default [1; 2 for ASYNC runs of one graph with slots 1
                                 or 2]; 1: labels are vertex ids; 2: labels are
                                 positions in the reference GPU path's vertex order (degree
                                 partition, inc/rakLowmemCuda.hxx:505-519, 563), which its pickless
                                 rule compares; results are vertex ids either way; in a batch,
                                 each graph's own order. ASYNC runs, batches and the server take
                                 either; SYNC modes and graph steps label by id and refuse 2 */
  int64_t wait_timeout_ns;    /* 0: default [20 s]; bound on each device-side wait (the grid barrier
                                 between iterations). When it runs out the launch records
                                 RAK_ERR_TIMEOUT, every block leaves, and the call returns that
                                 status with the context still usable (the reference has no bound:
                                 a stuck kernel hangs its blocking read-back, inc/rakLowmemCuda.hxx
                                 :486, and errors exit(), inc/_cuda.hxx:221-235) */
  int32_t tie_break;          /* -1 or 0: mode default; 1: the reference's tie rule for Misra-Gries
                                 sketches (inc/rakLowmem.hxx:164-171: the first slot of maximum
                                 weight, which is the most recently inserted key); 2: on iterations
                                 l < tie_iterations a maximum shared by several slots goes to the
                                 key with the largest hash of (vertex, key, l) (SplitMix64), then
                                 the reference's rule. CPU sketch rules only. ASYNC: 2 [2]; SYNC
                                 and SYNC_SPLIT: 1 [1], 2 on request (deterministic) */
  int32_t tie_iterations;     /* 0: default [2]; iterations with hashed ties under tie_break 2 */
  int32_t edge_staging;       /* -1 or 0: default; 1: vertices and split-vertex chunks that a whole
                                 warp scans read their edges from shared-memory tiles filled by bulk
                                 copies (TMA, cp.async.bulk); 2: every lane loads its edges from
                                 global memory. Results are the same either way. [2] */
  int32_t max_blocks;         /* 0: as many thread blocks as fit on the device; k > 0: the persistent
                                 launch uses at most k blocks of 256 threads (fewer vertices in
                                 flight at once; leaves SMs to other work) [0] */
  int32_t dense_pct;          /* -1: never; 0: default [-1]; k in 1..100: asynchronous runs of one
                                 graph replace the pruned frontier by every vertex after heavy
                                 iterations: when the vertices that moved in an iteration hold at
                                 least k% of the edges, the next iteration's moves mark no
                                 neighbours and the iteration after it processes every vertex. The
                                 reference marks neighbours after every move (inc/rakCuda.hxx:96-103,
                                 called at inc/rakLowmemCuda.hxx:155,225,313,413) */
  int32_t renumber;           /* -1 or 0: default (1 for asynchronous runs on resident graphs --
                                 rak_graph_run -- of 2^22 vertices or more and average degree 8 or
                                 more, which pay for the copy once; otherwise 2); 1: the run works
                                 on a copy of the graph
                                 renumbered in the library's work order (heaviest vertices first),
                                 built on the device once per resident graph and layout; labels keep
                                 their values (vertex ids) and results come back in the graph's own
                                 numbering; RAK_MODE_ASYNC (either label order) and
                                 RAK_MODE_SYNC_SPLIT (whose results equal those on the graph as
                                 given). 2: on the graph as given. The reference runs on a copy in
                                 its own degree-partition order (inc/rakLowmemCuda.hxx:505-519,
                                 563-568) */
  int64_t reserved[3];
} rak_options;

typedef struct rak_result {
  int32_t iterations;          /* RakResult::iterations */
  float time_ms;               /* RakResult::time: init + mark + iterations, device time, averaged */
  float marking_time_ms;       /* RakResult::markingTime */
  float initialization_time_ms;/* RakResult::initializationTime */
  float memory_gb;             /* RakResult::memory: working buffers beyond the graph, in GB */
  float plan_ms;               /* degree bucketing of the graph on the device (once per graph) */
  float h2d_ms;                /* host->device copies inside this call (host-located csr) */
  float d2h_ms;                /* device->host copy of the membership (host-located csr) */
  uint64_t peak_device_bytes;  /* all device memory this call held at once, graph included */
  uint64_t traversed_edges;    /* sum over iterations of the degrees of the vertices processed */
  uint64_t processed_vertices; /* sum over iterations of the vertices processed */
  uint64_t changed_last;       /* vertices that changed label in the last iteration */
  uint64_t moved_vertices;     /* sum over iterations of the vertices that changed label */
  uint64_t moved_edges;        /* sum over iterations of the degrees of the vertices that moved */
  float loop_ms;               /* device time of the iterations alone (the persistent kernel) */
  float reserved_f;
  double modularity;           /* when requested, else NaN */
  uint64_t marked_edges;       /* sum over iterations of the degrees of the moved vertices whose
                                  neighbours were marked (moved_edges less the dense iterations'
                                  moves, rak_options.dense_pct) */
  int32_t dense_iterations;    /* iterations whose moves marked no neighbours (dense_pct) */
  int32_t reserved_r;
} rak_result;

typedef struct rak_ctx rak_ctx;
typedef struct rak_graph rak_graph;

/* ---- library ---------------------------------------------------------------------------- */
int rak_abi_version(void);
const char *rak_status_string(rak_status s);
/* Fills the defaults documented above. */
void rak_options_default(rak_options *o);

/* ---- context ---------------------------------------------------------------------------- */
/* Binds to `device` (must be sm_100). No reference counterpart: the reference uses the default
 * device and stream (inc/rakLowmemCuda.hxx:570). */
rak_status rak_ctx_create(int device, rak_ctx **out);
rak_status rak_ctx_destroy(rak_ctx *ctx);
/* Work is issued on `stream` (a cudaStream_t; NULL = the context's own stream). */
rak_status rak_ctx_set_stream(rak_ctx *ctx, void *stream);
/* Device memory the context keeps mapped between rak_lowmem_cuda calls (default 0: every call
 * releases what it allocated, as the reference does). With bytes > 0 the call's graph copy and
 * working buffers come from a stream-ordered pool of the context that keeps up to `bytes` after
 * the call, so repeated calls on graphs of similar size skip mapping and unmapping them.
 * No reference counterpart. */
rak_status rak_ctx_set_memory_keep(rak_ctx *ctx, uint64_t bytes);
/* Text of the last error on this context (empty if none). */
const char *rak_ctx_last_error(const rak_ctx *ctx);

/* ---- single graph ----------------------------------------------------------------------- */
/* rakLowmemStaticCuda<SLOTS>(x, o) / rakLowmemInvokeCuda(x, o, fi, fm): one complete run.
 * q: initial labels (NULL: identity, as rakInitializeCuW does, inc/rakCuda.hxx:25-44), n entries.
 * membership: n entries, written. q and membership are in g->location. Host graphs are copied
 * to the device inside the call (h2d_ms) and freed before returning, as the reference does. */
rak_status rak_lowmem_cuda(rak_ctx *ctx, const rak_csr *g, const uint32_t *q,
                           const rak_options *o, uint32_t *membership, rak_result *res);

/* Makes a device-resident copy of g (or binds a device-located g without copying) and builds
 * its degree-bucket plan for the layout in o (NULL: defaults). */
rak_status rak_graph_create(rak_ctx *ctx, const rak_csr *g, const rak_options *o, rak_graph **out);
rak_status rak_graph_destroy(rak_graph *gr);
/* Device bytes held by the resident graph (copy + plan). */
uint64_t rak_graph_device_bytes(const rak_graph *gr);

/* A complete run on a resident graph. q (may be NULL) and membership are device pointers. */
rak_status rak_graph_run(rak_ctx *ctx, rak_graph *gr, const uint32_t *q, const rak_options *o,
                         uint32_t *membership, rak_result *res);

/* One move iteration with index `iteration` (pickless schedule) from the snapshot
 * (vcom_prev, aff_prev) into (vcom_next, aff_next); all device pointers, n entries each.
 * In RAK_MODE_ASYNC the update is in place on vcom_next/aff_next after copying prev into them.
 * *changed receives the number of vertices that changed label. */
rak_status rak_graph_step(rak_ctx *ctx, rak_graph *gr, const rak_options *o, int iteration,
                          const uint32_t *vcom_prev, const uint8_t *aff_prev,
                          uint32_t *vcom_next, uint8_t *aff_next, uint64_t *changed);

/* modularityBy(x, membership, M=w(x)/2, R=1) accumulated in FP64 on the device.
 * membership is in g->location. */
rak_status rak_modularity_f64(rak_ctx *ctx, const rak_csr *g, const uint32_t *membership,
                              double *q);

/* ---- batches of independent graphs ------------------------------------------------------- */
/* Many graphs concatenated into one CSR: graph g owns vertices [graph_offsets[g],
 * graph_offsets[g+1]); offsets index the concatenated targets/weights; targets are ids LOCAL to the
 * edge's own graph. Replaces a loop of rakLowmemStaticCuda calls, one per graph (main.cxx:84-92). */
typedef struct rak_batch_csr {
  int64_t graphs;                /* number of graphs */
  int64_t n;                     /* total vertices, == graph_offsets[graphs], < 2^31 */
  int64_t m;                     /* total directed edges, == offsets[n] */
  int32_t location;              /* rak_location of every array */
  int32_t reserved;
  const int64_t *graph_offsets;  /* graphs+1 */
  const int64_t *offsets;        /* n+1 */
  const uint32_t *targets;       /* m local ids */
  const float *weights;          /* m, or NULL for unit weights */
} rak_batch_csr;

typedef struct rak_batch rak_batch;

/* Device-resident copy of a batch (or a binding of a device-located one) with its plan. */
rak_status rak_batch_create(rak_ctx *ctx, const rak_batch_csr *b, const rak_options *o, rak_batch **out);
rak_status rak_batch_destroy(rak_batch *b);
/* Enqueues one complete run of every graph on the context's stream -- a single persistent launch
 * in which each graph iterates until its own convergence test passes -- and returns without
 * waiting. q (local initial labels, may be NULL) and membership (local labels, written) are device
 * pointers with n entries. The sequence makes no host round trip, so it can be captured into a
 * CUDA graph. */
rak_status rak_batch_launch(rak_ctx *ctx, rak_batch *b, const uint32_t *q, const rak_options *o,
                            uint32_t *membership);
/* Waits for the last launch; iterations (host, `graphs` entries, may be NULL) receives each graph's
 * iteration count, total (may be NULL) the counters summed over graphs. */
rak_status rak_batch_results(rak_ctx *ctx, rak_batch *b, int32_t *iterations, rak_result *total);
/* Captures rak_batch_launch(q, o, membership) into a CUDA graph kept by the batch, and replays it. */
rak_status rak_batch_capture(rak_ctx *ctx, rak_batch *b, const uint32_t *q, const rak_options *o,
                             uint32_t *membership);
rak_status rak_batch_replay(rak_ctx *ctx, rak_batch *b);
/* FP64 modularity of every graph (membership: device, local labels); q: host, `graphs` entries. */
rak_status rak_batch_modularity_f64(rak_ctx *ctx, rak_batch *b, const uint32_t *membership, double *q);

/* ---- autotuning ------------------------------------------------------------------------------ */
/* Picks lane_max / hub_min (degree thresholds), hub_chunk (the split-vertex tile) and slots (MG
 * slot count) by running the graph or batch: coordinate descent from `base` over the values in the
 * space, one dimension at a time, keeping the fastest run to convergence whose FP64 modularity
 * (the mean over graphs for a batch) is at least Q_base * (1 - quality_rel) - quality_abs.
 * No reference counterpart (the reference fixes these at compile time). */
typedef struct rak_tune_space {
  int32_t lane_max[8];  int32_t n_lane_max;   /* [32 64 128 256] */
  int32_t hub_min[8];   int32_t n_hub_min;    /* [4096 8192 16384 32768 65536] */
  int32_t hub_chunk[8]; int32_t n_hub_chunk;  /* [2048 4096 8192 16384] */
  int32_t slots[5];     int32_t n_slots;      /* [4 8 16] */
  int32_t repeats;                            /* timed runs per candidate, best kept [2] */
  int32_t label_orders;                       /* 1: asynchronous runs also try the other label
                                                 order (ids / reference order), first [1] */
  double quality_rel, quality_abs;            /* [0.005, 0.001] */
} rak_tune_space;

typedef struct rak_tune_entry {  /* one candidate that was run */
  int32_t lane_max, hub_min, hub_chunk, slots;
  int32_t iterations, accepted;  /* accepted: passed the quality gate */
  int32_t label_order, reserved; /* label order of the run (1 ids, 2 reference order) */
  double ms;                     /* best time to result */
  double modularity;
  double edges_per_s;            /* traversed edges per second of that run */
} rak_tune_entry;

void rak_tune_space_default(rak_tune_space *sp);
/* membership: device buffer of the graph's n labels, used by the runs. log (may be NULL) receives
 * up to log_cap entries; *log_len (may be NULL) the number of candidates run. */
rak_status rak_graph_autotune(rak_ctx *ctx, rak_graph *gr, const rak_options *base, const rak_tune_space *space,
                              uint32_t *membership, rak_options *best, rak_tune_entry *log, int32_t log_cap,
                              int32_t *log_len);
/* The same for a batch of `graphs` graphs (membership: device, the batch's n labels). */
rak_status rak_batch_autotune(rak_ctx *ctx, rak_batch *b, int64_t graphs, const rak_options *base,
                              const rak_tune_space *space, uint32_t *membership, rak_options *best,
                              rak_tune_entry *log, int32_t log_cap, int32_t *log_len);

/* ---- serving: continuous batching of requests --------------------------------------------- */
/* A request loop (its own host thread) that keeps admitted graphs resident on the device, admits
 * waiting requests as soon as device-memory budget and a launch slot are free, packs them into a
 * batch and runs it as one persistent launch; several launches run at once on separate streams
 * (each capped to its share of the SMs), so requests that arrive while others are on the GPU
 * overlap with them. No reference counterpart (the reference runs one graph per call). */
typedef struct rak_server rak_server;

typedef struct rak_server_options {
  uint64_t budget_bytes;        /* device bytes for admitted requests (graphs + working buffers) */
  int32_t max_graphs_per_launch;/* requests packed into one launch at most [256] */
  int32_t slots;                /* launches in flight at once, each on its own stream [2] */
  int32_t queue_capacity;       /* waiting requests before submit returns RAK_ERR_BUSY [65536] */
  int32_t reserved;
  rak_options run;              /* options of every run (layout, mode, slots, tolerance, ...) */
} rak_server_options;

typedef struct rak_server_stats {
  uint64_t submitted, completed, rejected, launches, graphs_launched;
  uint64_t edges_completed;     /* directed edges of completed requests */
  uint64_t device_bytes_in_use; /* budget currently held by admitted requests */
  int32_t max_concurrent_launches;
  int32_t pending;              /* requests waiting for admission */
  double load_ms;               /* host time packing and uploading launches, plan included (summed) */
  double plan_ms;               /* of which building the plan on the device (summed) */
  double run_ms;                /* launch-to-completion time of launches (summed) */
  double pack_ms;               /* of load_ms: enqueueing uploads and the gather, checks included */
  double plan_host_ms;          /* of load_ms: building the plan, waits included */
  double enqueue_ms;            /* host time enqueueing the persistent launches (summed) */
} rak_server_stats;

void rak_server_options_default(rak_server_options *o);
/* Starts the loop on ctx's device. */
rak_status rak_server_create(rak_ctx *ctx, const rak_server_options *o, rak_server **out);
/* Queues a graph; its arrays must stay valid and unchanged until the request completes.
 * Host-located graphs are uploaded when their launch is packed (page-locked arrays copy fastest)
 * and, with run.validate, checked here on the caller's thread. Device-located graphs (on the
 * server's device: an arena of graphs kept in HBM) are packed by a device-to-device gather and,
 * with run.validate, checked on the device before their launch; a graph that fails ends with
 * RAK_ERR_INVALID_CSR from rak_server_wait. RAK_ERR_BUSY when the queue is full. */
rak_status rak_server_submit(rak_server *s, const rak_csr *g, uint64_t *ticket);
/* Waits up to timeout_s for a request (RAK_ERR_TIMEOUT otherwise), then copies its membership
 * (host, n entries; may be NULL) and result: iterations; time_ms = latency from submit to
 * completion; plan_ms = time waiting for admission. The ticket is released. A request larger than
 * the whole budget completes with RAK_ERR_OUT_OF_MEMORY. */
rak_status rak_server_wait(rak_server *s, uint64_t ticket, double timeout_s, uint32_t *membership,
                           rak_result *res);
rak_status rak_server_stats_get(rak_server *s, rak_server_stats *st);
/* Finishes every queued request, then stops the loop and frees everything. */
rak_status rak_server_destroy(rak_server *s);

/* ---- a run that allocates no device memory ------------------------------------------------ */
/* Size of the fixed device array rak_lowmem_cuda_noalloc works in. Every GPU that loads the
 * library holds this many bytes until the process exits. */
#define RAK_NOALLOC_SCRATCH_BYTES (64u << 20)

/* No counterpart in the reference (its runs allocate and free their buffers, inc/rakLowmemCuda.hxx
 * :570-605). For callers that cannot call cudaMalloc -- e.g. a process whose device memory is
 * already held by a framework's pooling allocator, or a latency-critical loop that must not pay
 * cudaMalloc/cudaFree's device synchronisation -- this runs rak_lowmem_cuda on a device-located
 * graph with every working buffer (flags, plan and its sort space, split-vertex tables and
 * partial sketches, counters) carved from one file-scope device array of
 * RAK_NOALLOC_SCRATCH_BYTES; it calls no cudaMalloc, cudaFree or allocating library routine.
 * g, q (may be NULL), o->initial_flags (may be NULL) and membership are device pointers; work is
 * issued on `stream` (a cudaStream_t, NULL = legacy default stream) of `device`.
 * Graphs whose buffers exceed the array (roughly 20 bytes per vertex, 28 with the reference label
 * order that asynchronous runs use by default, plus 8*slots bytes per split chunk) return
 * RAK_ERR_OUT_OF_MEMORY with res->peak_device_bytes set to the bytes needed. Options and labels
 * mean what they mean for rak_lowmem_cuda, except rak_options.renumber: runs here always work on
 * the graph as given (a renumbered copy would not fit the array).
 * The first call on a device looks the array up on that device (make it before any stream
 * capture). CUDA places the array, and each kernel variant's code (slot count, mode, offset width,
 * weighted or unit), on a device lazily, when a call first needs it; those are the runtime's own
 * device allocations, so a caller about to hand a device's memory to a pool makes one call of each
 * variant it will use first. All calls share the array and it keeps the last call's contents; each
 * call clears what must start at zero, and calls that overlap on the GPU race on it. Times in res
 * are host wall-clock (no CUDA events are created). The caller's current device is restored. */
rak_status rak_lowmem_cuda_noalloc(int device, void *stream, const rak_csr *g, const uint32_t *q,
                                   const rak_options *o, uint32_t *membership, rak_result *res);

/* ---- synthetic graphs (host, deterministic; for tests and benchmarks) -------------------- */
/* A host CSR allocated by the library; free with rak_host_csr_free. */
typedef struct rak_host_csr {
  int64_t n, m;
  int64_t *offsets;   /* n+1 */
  uint32_t *targets;  /* m */
  float *weights;     /* m, or NULL when unit weights were requested */
  uint32_t *truth;    /* planted labels (SBM), or NULL */
} rak_host_csr;

/* Symmetric R-MAT: n*edge_factor samples, each quadrant step chosen with probabilities
 * (a, b, c, 1-a-b-c); self-loops and duplicates removed, both directions stored. Weights are
 * uniform in [w_lo, w_hi) per undirected pair (same value both ways); w_lo == w_hi == 1 gives
 * NULL weights. threads <= 0: all cores. */
rak_status rak_gen_rmat(int scale, double edge_factor, double a, double b, double c, uint64_t seed,
                        float w_lo, float w_hi, int threads, rak_host_csr *out);
/* The same symmetric R-MAT built on ctx's device, bit-identical to rak_gen_rmat for the same
 * arguments (same samples, sorted duplicate-free adjacency, same weights; unit weights leave
 * weights NULL). offset_bits 32 or 64. Arrays are allocated on the device; free them with
 * rak_device_csr_free. Needs about 16 bytes of device memory per sampled edge direction while it
 * builds (a scale-27, edge-factor-16 graph: ~70 GB). No reference counterpart (the reference reads
 * its graphs from files). */
rak_status rak_gen_rmat_device(rak_ctx *ctx, int scale, double edge_factor, double a, double b, double c,
                               uint64_t seed, float w_lo, float w_hi, int32_t offset_bits, rak_csr *out);
/* The planted-partition SBM of rak_gen_sbm built on ctx's device, bit-identical to it (unit weights:
 * weights NULL; the planted block of vertex u is floor(u*k/n)). Needs about 16 bytes of device memory
 * per sampled edge direction while it builds. No reference counterpart. */
rak_status rak_gen_sbm_device(rak_ctx *ctx, int64_t n, int64_t k, double avg_degree, double in_out_ratio, uint64_t seed,
                              int32_t offset_bits, rak_csr *out);
rak_status rak_device_csr_free(rak_csr *g);
/* The vertex order the reference's GPU path works in (inc/rakLowmemCuda.hxx:505-519, 563: vertex
 * ids partitioned by degree < 4, then the rest by degree < 128, with libstdc++'s std::partition
 * exchange), whose positions name the labels of asynchronous runs (rak_options.label_order).
 * g device-located; ks: device, n entries (ks[i] = i-th vertex). */
rak_status rak_reference_vertex_order(rak_ctx *ctx, const rak_csr *g, uint32_t *ks);
/* The same order for every graph of a batch: ks (device, the batch's n entries) holds, in each
 * graph's range, that graph's local vertex ids in its reference order. */
rak_status rak_batch_reference_vertex_order(rak_ctx *ctx, rak_batch *b, uint32_t *ks);
/* Copies a device-located CSR into newly allocated host arrays (offsets widened to 64 bits); free
 * them with rak_host_csr_free. */
rak_status rak_device_csr_to_host(const rak_csr *g, rak_host_csr *out);
/* Planted-partition SBM: n vertices in k equal blocks, expected degree avg_degree, ratio
 * p_in/p_out; unit weights; truth[] holds the planted block of each vertex. */
rak_status rak_gen_sbm(int64_t n, int64_t k, double avg_degree, double in_out_ratio, uint64_t seed,
                       int threads, rak_host_csr *out);
/* 2D 4-neighbour lattice of width x height, each undirected edge deleted with probability
 * p_delete, plus shortcut_frac * (edges) random undirected shortcuts; unit weights. */
rak_status rak_gen_lattice(int64_t width, int64_t height, double p_delete, double shortcut_frac,
                           uint64_t seed, int threads, rak_host_csr *out);
/* Reads a Matrix Market coordinate file as the reference's driver does (inc/mtx.hxx
 * readMtxOmpW, inc/symmetrize.hxx symmetrizeOmpU, main.cxx:116-119): 1-based entries become 0-based
 * vertices (n = max(rows, cols)); "symmetric"/"skew-symmetric" files store both directions; with
 * weighted, the third column is the weight and 0 reads as 1 (else weights are NULL: unit); a
 * repeated (u, v) keeps its last occurrence in the file; with symmetrize, a missing reverse edge
 * is added with the same weight. threads <= 0: all cores. */
rak_status rak_read_mtx(const char *path, int weighted, int symmetrize, int threads, rak_host_csr *out);
void rak_host_csr_free(rak_host_csr *g);

/* Host-side CSR check (same rules as the device check): RAK_OK or RAK_ERR_INVALID_CSR. */
rak_status rak_csr_validate_host(const rak_csr *g);

/* Degree-bucket plan summary computed on the host from degrees (for tests and tooling):
 * fills counts[0..7] = vertices per lane group size 1,2,4,8,16,32, hubs, isolated, and returns
 * the number of hub chunks through *hub_chunks. */
rak_status rak_plan_summary_host(const rak_csr *g, const rak_options *o, int64_t counts[8],
                                 int64_t *hub_chunks);

#ifdef __cplusplus
}
#endif
#endif
