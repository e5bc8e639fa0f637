/*
 * rak_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's sketch-based label propagation (LPA) on the CPU,
 * used as the checker by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.
 * The product library never links, loads or calls anything in this directory.
 *
 * Parity is pinned two ways:
 *   - against the reference's own CPU code compiled from its sources into oracle/_ref/
 *     (oracle/ref_bridge.cpp, built by oracle/Makefile), and
 *   - against golden vectors generated from that build and committed under tests/golden/.
 *
 * Id space: vertices and labels are 0-based here. The reference's CPU code numbers vertices
 * from 1 (its MTX reader never creates vertex 0, mtx.hxx:213,238) and uses label 0 / key 0 as
 * "none"; this restatement uses ORC_NONE (0xFFFFFFFF) for "no key" instead, which is the same
 * rule shifted by one.
 */
#ifndef RAK_ORACLE_H
#define RAK_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NONE 0xFFFFFFFFu
#define ORC_MAX_SLOTS 32

/* A CSR graph held on the host. Weights may be NULL, meaning every edge weighs 1.0f. */
typedef struct orc_csr {
  int64_t n;
  const int64_t *off;   /* n+1 entries */
  const uint32_t *tgt;  /* off[n] entries */
  const float *wt;      /* off[n] entries or NULL */
} orc_csr;

/* How a vertex's edge list is divided among GPU lanes in the split per-vertex algorithm.
 *   deg <= lane_max            : one lane scans all edges in order (identical to the exact scan)
 *   lane_max < deg <= hub_min  : a group of G lanes, G the smallest power of two >= 2 with
 *                                G*lane_max >= deg, capped at 32; lane s takes edges s, s+G, ...
 *   deg > hub_min              : chunks of hub_chunk edges; lane s of 32 takes chunk edges
 *                                s, s+32, ...; chunk sketches merged in a fixed tree. */
typedef struct orc_layout {
  int64_t lane_max;
  int64_t hub_min;
  int64_t hub_chunk;
} orc_layout;

typedef struct orc_opts {
  int slots;              /* 1: weighted Boyer-Moore; 2..32: Misra-Gries with this many slots */
  int rescan;             /* Misra-Gries, exact scan only: recompute exact weights of the keys */
  int split;              /* 0: exact sequential scan of every vertex; 1: split layout above */
  orc_layout layout;
  double tolerance;       /* stop when changed/N <= tolerance */
  int max_iterations;
  int pickless_step;      /* iterations l with l % step == 0 only move to smaller labels; 0 = never */
  int check_on_pickless;  /* 0: the tolerance test is skipped on pickless iterations */
  int gpu_rule;           /* 0: the reference CPU sketch rules; 1: its GPU rules (first free slot,
                             no clamp, tournament argmax, move if w != 0, Boyer-Moore from the
                             vertex's own label) */
  int tie_until;          /* CPU rules, Misra-Gries: on iterations l < tie_until a maximum shared by
                             several slots goes to the key with the largest orc_tie_hash(u, key, l);
                             0: the reference's linear first maximum throughout */
} orc_opts;

typedef struct orc_sketch {
  uint32_t k[ORC_MAX_SLOTS];
  float w[ORC_MAX_SLOTS];
} orc_sketch;

/* Sketch primitives (exported for unit tests on hand-made edge streams). */
void orc_sketch_clear(orc_sketch *s, int slots);
void orc_mg_accumulate(orc_sketch *s, int slots, uint32_t c, float w);
void orc_bm_accumulate(orc_sketch *s, uint32_t c, float w);
void orc_sketch_merge(orc_sketch *a, const orc_sketch *b, int slots);
void orc_sketch_choose(const orc_sketch *s, int slots, uint32_t *c, float *w);
void orc_mg_accumulate_gpu(orc_sketch *s, int slots, uint32_t c, float w);
void orc_sketch_choose_gpu(const orc_sketch *s, int slots, uint32_t *c, float *w);

/* SplitMix64 finaliser (Steele, Lea & Flood, OOPSLA 2014) of (key << 32 | u) ^ l * 0xD6E8FEB86659FD93:
 * the tie order of the library's hashed ties (rak_options.tie_break 2). */
uint64_t orc_tie_hash(uint32_t u, uint32_t key, uint32_t l);
/* Largest weight; among equal maximum weights the key with the largest orc_tie_hash (lower slot on
 * equal hashes). */
void orc_sketch_choose_hashed(const orc_sketch *s, int slots, uint32_t u, uint32_t l, uint32_t *c, float *w);

/* Best label of vertex u given a label snapshot vcom (before the move rule is applied). */
void orc_choose(const orc_csr *g, const orc_opts *o, uint32_t u, const uint32_t *vcom,
                uint32_t *c, float *w);

/* One synchronous iteration: reads (vcom_prev, aff_prev), writes (vcom_next, aff_next).
 * aff_next is fully overwritten. Returns the number of vertices that changed label. */
uint64_t orc_sync_step(const orc_csr *g, const orc_opts *o, int iteration,
                       const uint32_t *vcom_prev, const uint8_t *aff_prev,
                       uint32_t *vcom_next, uint8_t *aff_next,
                       uint64_t *edges_out, uint64_t *processed_out);

/* Full synchronous run from labels q (NULL: identity), all vertices affected.
 * Writes final labels; returns iterations performed. */
int orc_sync_run(const orc_csr *g, const orc_opts *o, const uint32_t *q, uint32_t *labels,
                 uint64_t *edges_out);

/* The reference CPU loop run by one thread: in-place label and flag updates in vertex order,
 * and Misra-Gries keys carried from one vertex to the next as in a reused per-thread buffer. */
int orc_serial_run(const orc_csr *g, int slots, int rescan, double tolerance, int max_iterations,
                   uint32_t *labels);

/* FP64 modularity of a labelling (resolution 1). */
double orc_modularity(const orc_csr *g, const uint32_t *labels);

#ifdef __cplusplus
}
#endif
#endif
