/*
 * rak_oracle.c -- TEST INFRASTRUCTURE ONLY (see rak_oracle.h).
 *
 * CPU restatement of the reference's memory-efficient label propagation:
 *   - Misra-Gries accumulate          : inc/rakLowmem.hxx:63-89   (rakLowmemScanCommunityU)
 *   - exact rescan and argmax          : inc/rakLowmem.hxx:151-172 (rakLowmemChooseCommunityW)
 *   - weighted Boyer-Moore             : inc/rakLowmem.hxx:115-128 (rakLowmemScanCommunitiesMajority)
 *   - move rule, marking, loop         : inc/rakLowmem.hxx:189-212, 257-260
 *   - sketch merge by re-accumulation  : inc/sketchCuda.hxx:150-158 (sketchMergeWarpCudU)
 *   - pickless rule                    : inc/rakLowmemCuda.hxx:473-487
 *   - modularity                       : inc/properties.hxx:123-126, 177-192
 *   - GPU rule set (gpu_rule)          : inc/sketchCuda.hxx:73-108 (accumulate), 190-201 (argmax),
 *                                        inc/rakLowmemCuda.hxx:41-43, 152, 306 (BM start, moves)
 * Floating point follows the reference exactly: float sketch weights, adds and subtracts only
 * (no multiply, so no contraction), double modularity.
 */
#include "rak_oracle.h"
#include <stdlib.h>
#include <string.h>

static float edge_w(const orc_csr *g, int64_t e) { return g->wt ? g->wt[e] : 1.0f; }

void orc_sketch_clear(orc_sketch *s, int slots) {
  for (int i = 0; i < slots; ++i) { s->k[i] = ORC_NONE; s->w[i] = 0.0f; }
}

/* inc/rakLowmem.hxx:63-89: add w to every slot holding c; if none held it, the LAST slot whose
 * weight is zero takes (c, w); if no slot is free, every weight drops by w, clamped at zero. */
void orc_mg_accumulate(orc_sketch *s, int slots, uint32_t c, float w) {
  int has = 0;
  for (int i = 0; i < slots; ++i)
    if (s->k[i] == c) { s->w[i] += w; has = 1; }
  if (has) return;
  int f = -1;
  for (int i = 0; i < slots; ++i)
    if (s->w[i] == 0.0f) f = i;
  if (f >= 0) { s->k[f] = c; s->w[f] = w; return; }
  for (int i = 0; i < slots; ++i) {
    float t = s->w[i] - w;
    s->w[i] = t < 0.0f ? 0.0f : t;
  }
}

/* inc/sketchCuda.hxx:73-108 (sketchAccumulateWarpCudU, one sketch per thread): add w to every slot
 * holding c; if none held it, the FIRST slot whose weight is exactly zero takes (c, w); if no slot
 * is free, every weight drops by w, without a clamp. */
void orc_mg_accumulate_gpu(orc_sketch *s, int slots, uint32_t c, float w) {
  int has = 0;
  for (int i = 0; i < slots; ++i)
    if (s->k[i] == c) { s->w[i] += w; has = 1; }
  if (has) return;
  for (int i = 0; i < slots; ++i)
    if (s->w[i] == 0.0f) { s->k[i] = c; s->w[i] = w; return; }
  for (int i = 0; i < slots; ++i) s->w[i] -= w;
}

/* inc/sketchCuda.hxx:190-201: tournament -- at each level slot i takes slot i+ds when strictly
 * heavier; the winner is slot 0, whatever its weight. */
void orc_sketch_choose_gpu(const orc_sketch *s, int slots, uint32_t *c, float *w) {
  uint32_t k[ORC_MAX_SLOTS];
  float x[ORC_MAX_SLOTS];
  for (int i = 0; i < slots; ++i) { k[i] = s->k[i]; x[i] = s->w[i]; }
  for (int ds = slots / 2; ds >= 1; ds /= 2)
    for (int i = 0; i < ds; ++i)
      if (x[i + ds] > x[i]) { k[i] = k[i + ds]; x[i] = x[i + ds]; }
  *c = k[0]; *w = x[0];
}

/* inc/rakLowmem.hxx:120-126: weighted Boyer-Moore vote held in slot 0. */
void orc_bm_accumulate(orc_sketch *s, uint32_t c, float w) {
  if (c == s->k[0]) s->w[0] += w;
  else if (s->w[0] > w) s->w[0] -= w;
  else { s->k[0] = c; s->w[0] = w; }
}

static void acc_rule(orc_sketch *s, int slots, uint32_t c, float w, int gpu) {
  if (slots == 1) orc_bm_accumulate(s, c, w);
  else if (gpu) orc_mg_accumulate_gpu(s, slots, c, w);
  else orc_mg_accumulate(s, slots, c, w);
}

static void merge_rule(orc_sketch *a, const orc_sketch *b, int slots, int gpu) {
  for (int j = 0; j < slots; ++j)
    if (b->w[j] != 0.0f) acc_rule(a, slots, b->k[j], b->w[j], gpu);
}

/* inc/sketchCuda.hxx:150-158: merge b into a by re-accumulating b's non-zero slots in order. */
void orc_sketch_merge(orc_sketch *a, const orc_sketch *b, int slots) { merge_rule(a, b, slots, 0); }

/* inc/rakLowmem.hxx:164-171: linear argmax, strict '>', starting from weight 0. */
void orc_sketch_choose(const orc_sketch *s, int slots, uint32_t *c, float *w) {
  uint32_t cm = ORC_NONE;
  float wm = 0.0f;
  for (int i = 0; i < slots; ++i)
    if (s->w[i] > wm) { wm = s->w[i]; cm = s->k[i]; }
  *c = cm; *w = wm;
}

static uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

uint64_t orc_tie_hash(uint32_t u, uint32_t key, uint32_t l) {
  return mix64((((uint64_t)key << 32) | (uint64_t)u) ^ ((uint64_t)l * 0xD6E8FEB86659FD93ull));
}

void orc_sketch_choose_hashed(const orc_sketch *s, int slots, uint32_t u, uint32_t l, uint32_t *c, float *w) {
  uint32_t cm = ORC_NONE;
  float wm = 0.0f;
  uint64_t hb = 0;
  for (int i = 0; i < slots; ++i) {
    const uint64_t h = orc_tie_hash(u, s->k[i], l);
    if (s->w[i] > wm || (s->w[i] == wm && wm > 0.0f && h > hb)) { wm = s->w[i]; cm = s->k[i]; hb = h; }
  }
  *c = cm; *w = wm;
}

/* Sequential scan of edges [b, e) of u with stride st (self-loops skipped, rakLowmem.hxx:65). */
static void scan_range(const orc_csr *g, uint32_t u, const uint32_t *vcom, int slots,
                       int64_t b, int64_t e, int64_t st, orc_sketch *s, int gpu) {
  for (int64_t i = b; i < e; i += st) {
    uint32_t v = g->tgt[i];
    if (v == u) continue;
    acc_rule(s, slots, vcom[v], edge_w(g, i), gpu);
  }
}

/* Fixed binary tree over lanes L[0..n): at each level lane s (< off) merges lane s+off. */
static void tree_merge(orc_sketch *L, int n, int slots, int gpu) {
  for (int off = n / 2; off >= 1; off /= 2)
    for (int s = 0; s < off; ++s) merge_rule(&L[s], &L[s + off], slots, gpu);
}

/* A cleared sketch; Boyer-Moore under the GPU rules starts from the vertex's own label d with
 * weight 0 (inc/rakLowmemCuda.hxx:41-43). */
static void clear_rule(orc_sketch *s, int slots, int gpu, uint32_t d) {
  orc_sketch_clear(s, slots);
  if (gpu && slots == 1) s->k[0] = d;
}

static int group_size(const orc_layout *ly, int64_t deg) {
  int G = 2;
  while (G < 32 && (int64_t)G * ly->lane_max < deg) G *= 2;
  return G;
}

/* The split per-vertex sketch (documented in rak_oracle.h, orc_layout). */
static void split_sketch(const orc_csr *g, const orc_opts *o, uint32_t u, const uint32_t *vcom,
                         orc_sketch *out) {
  const int S = o->slots, gpu = o->gpu_rule;
  const uint32_t d = vcom[u];
  const int64_t b = g->off[u], deg = g->off[u + 1] - g->off[u];
  const orc_layout *ly = &o->layout;
  orc_sketch L[32];
  if (deg <= ly->lane_max) {
    clear_rule(out, S, gpu, d);
    scan_range(g, u, vcom, S, b, b + deg, 1, out, gpu);
    return;
  }
  if (deg <= ly->hub_min) {
    int G = group_size(ly, deg);
    for (int s = 0; s < G; ++s) {
      clear_rule(&L[s], S, gpu, d);
      scan_range(g, u, vcom, S, b + s, b + deg, G, &L[s], gpu);
    }
    tree_merge(L, G, S, gpu);
    *out = L[0];
    return;
  }
  const int64_t CH = ly->hub_chunk, nch = (deg + CH - 1) / CH;
  orc_sketch *C = (orc_sketch *)malloc(sizeof(orc_sketch) * (size_t)nch);
  for (int64_t j = 0; j < nch; ++j) {
    int64_t cb = b + j * CH, ce = cb + CH < b + deg ? cb + CH : b + deg;
    for (int s = 0; s < 32; ++s) {
      clear_rule(&L[s], S, gpu, d);
      scan_range(g, u, vcom, S, cb + s, ce, 32, &L[s], gpu);
    }
    tree_merge(L, 32, S, gpu);
    C[j] = L[0];
  }
  for (int l = 0; l < 32; ++l) {
    clear_rule(&L[l], S, gpu, d);
    for (int64_t j = l; j < nch; j += 32) merge_rule(&L[l], &C[j], S, gpu);
  }
  tree_merge(L, 32, S, gpu);
  *out = L[0];
  free(C);
}

/* inc/rakLowmem.hxx:154-162: exact weights of the sketch keys, summed in edge order. */
static void rescan(const orc_csr *g, uint32_t u, const uint32_t *vcom, int slots, orc_sketch *s) {
  for (int i = 0; i < slots; ++i) s->w[i] = 0.0f;
  for (int64_t e = g->off[u]; e < g->off[u + 1]; ++e) {
    uint32_t v = g->tgt[e];
    if (v == u) continue;
    uint32_t c = vcom[v];
    float w = edge_w(g, e);
    for (int i = 0; i < slots; ++i)
      if (s->k[i] == c) s->w[i] += w;
  }
}

/* The per-vertex choice on iteration l (l < 0: outside any iteration, no hashed ties). */
static void choose_at(const orc_csr *g, const orc_opts *o, uint32_t u, const uint32_t *vcom, int l,
                      uint32_t *c, float *w) {
  orc_sketch s;
  if (o->split) {
    split_sketch(g, o, u, vcom, &s);
  } else {
    clear_rule(&s, o->slots, o->gpu_rule, vcom[u]);
    scan_range(g, u, vcom, o->slots, g->off[u], g->off[u + 1], 1, &s, o->gpu_rule);
    if (o->rescan && o->slots > 1) rescan(g, u, vcom, o->slots, &s);
  }
  if (o->gpu_rule) orc_sketch_choose_gpu(&s, o->slots, c, w);
  else if (o->slots > 1 && l >= 0 && l < o->tie_until) orc_sketch_choose_hashed(&s, o->slots, u, (uint32_t)l, c, w);
  else orc_sketch_choose(&s, o->slots, c, w);
}

void orc_choose(const orc_csr *g, const orc_opts *o, uint32_t u, const uint32_t *vcom,
                uint32_t *c, float *w) {
  choose_at(g, o, u, vcom, -1, c, w);
}

static int is_pickless(const orc_opts *o, int l) { return o->pickless_step > 0 && l % o->pickless_step == 0; }

/* Synchronous form of inc/rakLowmem.hxx:189-212: every decision reads the snapshot; a moved
 * vertex marks its neighbours other than itself (the reference marks, then clears u). */
uint64_t orc_sync_step(const orc_csr *g, const orc_opts *o, int iteration,
                       const uint32_t *vcom_prev, const uint8_t *aff_prev,
                       uint32_t *vcom_next, uint8_t *aff_next,
                       uint64_t *edges_out, uint64_t *processed_out) {
  const int pl = is_pickless(o, iteration);
  uint64_t changed = 0, edges = 0, processed = 0;
  memset(aff_next, 0, (size_t)g->n);
  for (int64_t u = 0; u < g->n; ++u) vcom_next[u] = vcom_prev[u];
  /* Every decision reads only the snapshot, so vertices are independent and may be decided by
   * several threads (OpenMP; one thread gives the same result). Marks are idempotent stores. */
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : changed, edges, processed)
  for (int64_t u = 0; u < g->n; ++u) {
    if (!aff_prev[u]) continue;
    int64_t deg = g->off[u + 1] - g->off[u];
    if (deg == 0) continue;
    ++processed; edges += (uint64_t)deg;
    uint32_t d = vcom_prev[u], c; float w;
    choose_at(g, o, (uint32_t)u, vcom_prev, iteration, &c, &w);
    /* CPU rule: w > 0; GPU rule: w != 0 for Misra-Gries, any candidate for Boyer-Moore */
    const int weight_ok = o->gpu_rule ? (o->slots == 1 || w != 0.0f) : (w > 0.0f);
    if (!weight_ok || c == d) continue;
    if (pl && c > d) continue;
    vcom_next[u] = c; ++changed;
    for (int64_t e = g->off[u]; e < g->off[u + 1]; ++e)
      if (g->tgt[e] != (uint32_t)u) __atomic_store_n(&aff_next[g->tgt[e]], (uint8_t)1, __ATOMIC_RELAXED);
  }
  if (edges_out) *edges_out += edges;
  if (processed_out) *processed_out += processed;
  return changed;
}

/* Loop of inc/rakLowmem.hxx:257-260 (tolerance test every iteration) with the optional
 * pickless schedule of inc/rakLowmemCuda.hxx:473-487. */
int orc_sync_run(const orc_csr *g, const orc_opts *o, const uint32_t *q, uint32_t *labels,
                 uint64_t *edges_out) {
  size_t n = (size_t)g->n;
  uint32_t *a = (uint32_t *)malloc(n * 4 + 4), *b = (uint32_t *)malloc(n * 4 + 4);
  uint8_t *fa = (uint8_t *)malloc(n + 1), *fb = (uint8_t *)malloc(n + 1);
  for (size_t u = 0; u < n; ++u) { a[u] = q ? q[u] : (uint32_t)u; fa[u] = 1; }
  int l = 0;
  while (l < o->max_iterations) {
    uint64_t ch = orc_sync_step(g, o, l, a, fa, b, fb, edges_out, NULL);
    uint32_t *t = a; a = b; b = t;
    uint8_t *tf = fa; fa = fb; fb = tf;
    int pl = is_pickless(o, l);
    ++l;
    if ((!pl || o->check_on_pickless) && (double)ch / (double)g->n <= o->tolerance) break;
  }
  memcpy(labels, a, n * 4);
  free(a); free(b); free(fa); free(fb);
  return l;
}

/* inc/rakLowmem.hxx:189-212 and 228-264 with one thread: in-place updates in vertex order.
 * Keys persist across vertices (the reference reuses one key array per thread and clears only
 * the weights, rakLowmem.hxx:200); the first vertex starts from keys that match nothing. */
int orc_serial_run(const orc_csr *g, int slots, int rescan_on, double tolerance, int max_iterations,
                   uint32_t *labels) {
  size_t n = (size_t)g->n;
  uint8_t *aff = (uint8_t *)malloc(n + 1);
  for (size_t u = 0; u < n; ++u) { labels[u] = (uint32_t)u; aff[u] = 1; }
  orc_sketch s;
  orc_sketch_clear(&s, ORC_MAX_SLOTS);
  int l = 0;
  for (l = 0; l < max_iterations;) {
    uint64_t a = 0;
    for (int64_t u = 0; u < g->n; ++u) {
      if (!aff[u]) continue;
      uint32_t d = labels[u], c; float w;
      if (slots > 1) {
        for (int i = 0; i < slots; ++i) s.w[i] = 0.0f;
        scan_range(g, (uint32_t)u, labels, slots, g->off[u], g->off[u + 1], 1, &s, 0);
        if (rescan_on) rescan(g, (uint32_t)u, labels, slots, &s);
        orc_sketch_choose(&s, slots, &c, &w);
      } else {
        orc_sketch bm; orc_sketch_clear(&bm, 1);
        scan_range(g, (uint32_t)u, labels, 1, g->off[u], g->off[u + 1], 1, &bm, 0);
        c = bm.k[0]; w = bm.w[0];
      }
      if (w > 0.0f && c != d) {
        labels[u] = c; ++a;
        for (int64_t e = g->off[u]; e < g->off[u + 1]; ++e) aff[g->tgt[e]] = 1;
      }
      aff[u] = 0;
    }
    ++l;
    if ((double)a / (double)g->n <= tolerance) break;
  }
  free(aff);
  return l;
}

/* inc/properties.hxx:177-192 (per-edge cin/ctot in vertex then edge order) and :123-126. */
double orc_modularity(const orc_csr *g, const uint32_t *labels) {
  size_t n = (size_t)g->n;
  double *cin = (double *)calloc(n + 1, sizeof(double)), *ctot = (double *)calloc(n + 1, sizeof(double));
  double m2 = 0.0;
  for (int64_t u = 0; u < g->n; ++u) {
    uint32_t c = labels[u];
    for (int64_t e = g->off[u]; e < g->off[u + 1]; ++e) {
      double w = (double)edge_w(g, e);
      if (labels[g->tgt[e]] == c) cin[c] += w;
      ctot[c] += w;
      m2 += w;
    }
  }
  double q = 0.0;
  if (m2 > 0.0)
    for (size_t c = 0; c < n; ++c) {
      double t = ctot[c] / m2;
      q += cin[c] / m2 - t * t;
    }
  free(cin); free(ctot);
  return q;
}
