/*
 * rmat_gen.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C (OpenMP) restatement of the library's deterministic synthetic graphs: the symmetric
 * R-MAT of rak_gen_rmat and the perturbed 2D lattice of rak_gen_lattice. It lets bench.py's
 * reference arm build its workload graph without loading the library, so that arm runs the
 * reference's CPU code and nothing of the product. tests/test_oracle_gen.py checks both
 * generators bit for bit (offsets, targets, weights) against the library's.
 *
 * Every random choice is word i of a counter-based stream: SplitMix64's finaliser (Steele, Lea &
 * Flood, OOPSLA 2014) applied to (a per-(seed, stream) key + i). A graph is built from samples
 * (u, v): both directions of each sample that is kept and is not a self-loop are stored, each
 * adjacency list is sorted and duplicates are dropped. Results do not depend on the thread count.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { STREAM_RMAT = 1, STREAM_WEIGHT = 2, STREAM_LATTICE = 4 };

typedef struct og_graph {
  int64_t n, m;
  int64_t *off;  /* n+1 */
  uint32_t *tgt; /* m */
  float *wt;     /* m, or NULL (unit weights) */
} og_graph;

static inline uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
/* rand64(seed, stream, i) == mix64(stream_key(seed, stream) + i) */
static inline uint64_t stream_key(uint64_t seed, uint64_t stream) {
  return mix64(seed ^ (stream * 0xD6E8FEB86659FD93ull));
}
static inline uint32_t below(uint64_t h, uint64_t n) { return (uint32_t)(((h >> 32) * n) >> 32); }

/* The sample of one generator: sample i gives (u, v), or is dropped (returns 0). */
typedef struct gen {
  int kind; /* 0: R-MAT, 1: lattice */
  /* R-MAT */
  int scale;
  uint64_t krmat;
  uint32_t tA, tAB, tABC;
  /* lattice */
  int64_t width, n, eh, grid;
  uint32_t del24;
  uint64_t klat, klat2;
} gen;

static inline int sample(const gen *g, int64_t i, uint32_t *u, uint32_t *v) {
  if (g->kind == 0) {
    /* each level takes 16 random bits; quadrant (0,0) with probability a, (0,1) b, (1,0) c, (1,1) d */
    uint32_t uu = 0, vv = 0;
    uint64_t h = 0;
    for (int L = 0; L < g->scale; ++L) {
      if ((L & 3) == 0) h = mix64(g->krmat + (uint64_t)i * 8 + (uint64_t)(L >> 2));
      const uint32_t r = (uint32_t)(h >> (16 * (L & 3))) & 0xFFFFu;
      const uint32_t ub = r >= g->tAB;
      const uint32_t vb = (r >= g->tA && r < g->tAB) || r >= g->tABC;
      uu = (uu << 1) | ub;
      vv = (vv << 1) | vb;
    }
    *u = uu;
    *v = vv;
    return 1;
  }
  /* lattice: horizontal edges, then vertical edges (each dropped with probability p_delete),
   * then uniform random shortcuts */
  const uint64_t h = mix64(g->klat + (uint64_t)i);
  if (i < g->grid) {
    if ((uint32_t)(h >> 40) < g->del24) return 0;
    if (i < g->eh) {
      const int64_t y = i / (g->width - 1), x = i % (g->width - 1);
      *u = (uint32_t)(y * g->width + x);
      *v = *u + 1;
    } else {
      const int64_t j = i - g->eh;
      *u = (uint32_t)j;
      *v = (uint32_t)(j + g->width);
    }
    return 1;
  }
  *u = below(h, (uint64_t)g->n);
  *v = below(mix64(g->klat2 + (uint64_t)i), (uint64_t)g->n);
  return 1;
}

static void insertion_sort(uint32_t *a, int64_t len) {
  for (int64_t i = 1; i < len; ++i) {
    const uint32_t x = a[i];
    int64_t j = i - 1;
    while (j >= 0 && a[j] > x) { a[j + 1] = a[j]; --j; }
    a[j + 1] = x;
  }
}

/* LSD radix sort of a[0..len) (values < 2^bits) with 8-bit digits through tmp. */
static void radix_sort(uint32_t *a, uint32_t *tmp, int64_t len, int bits) {
  int64_t cnt[256];
  uint32_t *src = a, *dst = tmp;
  for (int sh = 0; sh < bits; sh += 8) {
    memset(cnt, 0, sizeof(cnt));
    for (int64_t i = 0; i < len; ++i) ++cnt[(src[i] >> sh) & 255u];
    int64_t s = 0;
    for (int d = 0; d < 256; ++d) { const int64_t c = cnt[d]; cnt[d] = s; s += c; }
    for (int64_t i = 0; i < len; ++i) dst[cnt[(src[i] >> sh) & 255u]++] = src[i];
    uint32_t *t = src; src = dst; dst = t;
  }
  if (src != a) memcpy(a, src, (size_t)len * 4);
}

static int64_t sort_unique(uint32_t *a, int64_t len, uint32_t **tmp, int64_t *cap, int bits) {
  if (len <= 1) return len;
  if (len <= 64) {
    insertion_sort(a, len);
  } else {
    if (*cap < len) {
      free(*tmp);
      *tmp = (uint32_t *)malloc((size_t)len * 4);
      *cap = *tmp ? len : 0;
      if (!*tmp) return -1;
    }
    radix_sort(a, *tmp, len, bits);
  }
  int64_t k = 1;
  for (int64_t i = 1; i < len; ++i)
    if (a[i] != a[k - 1]) a[k++] = a[i];
  return k;
}

/* Symmetric CSR with sorted, duplicate-free adjacency and no self-loops from samples
 * [0, samples). Returns 0, or -1 when memory runs out. */
static int build_symmetric(const gen *g, int64_t n, int64_t samples, og_graph *out) {
  uint32_t *cnt = (uint32_t *)calloc((size_t)n + 1, 4);
  int64_t *off = (int64_t *)malloc(((size_t)n + 1) * 8);
  int64_t *cur = (int64_t *)malloc(((size_t)n + 1) * 8);
  if (!cnt || !off || !cur) { free(cnt); free(off); free(cur); return -1; }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < samples; ++i) {
    uint32_t u, v;
    if (!sample(g, i, &u, &v) || u == v) continue;
    __atomic_fetch_add(&cnt[u], 1u, __ATOMIC_RELAXED);
    __atomic_fetch_add(&cnt[v], 1u, __ATOMIC_RELAXED);
  }
  off[0] = 0;
  for (int64_t u = 0; u < n; ++u) off[u + 1] = off[u] + cnt[u];
  const int64_t raw = off[n];
  uint32_t *tmp = (uint32_t *)malloc((size_t)(raw > 0 ? raw : 1) * 4);
  if (!tmp) { free(cnt); free(off); free(cur); return -1; }
  memcpy(cur, off, (size_t)n * 8);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < samples; ++i) {
    uint32_t u, v;
    if (!sample(g, i, &u, &v) || u == v) continue;
    tmp[__atomic_fetch_add(&cur[u], (int64_t)1, __ATOMIC_RELAXED)] = v;
    tmp[__atomic_fetch_add(&cur[v], (int64_t)1, __ATOMIC_RELAXED)] = u;
  }
  free(cur);
  int bits = 1;
  while (bits < 32 && ((int64_t)1 << bits) < n) ++bits;
  int failed = 0;
#pragma omp parallel reduction(| : failed)
  {
    uint32_t *buf = NULL;
    int64_t cap = 0;
#pragma omp for schedule(dynamic, 1024)
    for (int64_t u = 0; u < n; ++u) {
      const int64_t k = sort_unique(tmp + off[u], off[u + 1] - off[u], &buf, &cap, bits);
      if (k < 0) failed = 1;
      else cnt[u] = (uint32_t)k;
    }
    free(buf);
  }
  if (failed) { free(cnt); free(off); free(tmp); return -1; }
  out->n = n;
  out->off = (int64_t *)malloc(((size_t)n + 1) * 8);
  if (!out->off) { free(cnt); free(off); free(tmp); return -1; }
  out->off[0] = 0;
  for (int64_t u = 0; u < n; ++u) out->off[u + 1] = out->off[u] + cnt[u];
  out->m = out->off[n];
  out->tgt = (uint32_t *)malloc((size_t)(out->m > 0 ? out->m : 1) * 4);
  if (!out->tgt) { free(cnt); free(off); free(tmp); free(out->off); out->off = NULL; return -1; }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < n; ++u)
    memcpy(out->tgt + out->off[u], tmp + off[u], (size_t)cnt[u] * 4);
  free(tmp);
  free(off);
  free(cnt);
  out->wt = NULL;
  return 0;
}

static void set_threads(int threads) {
  if (threads > 0) omp_set_num_threads(threads);
}

void og_free(og_graph *g) {
  if (!g) return;
  free(g->off);
  free(g->tgt);
  free(g->wt);
  memset(g, 0, sizeof(*g));
}

/* The library's rak_gen_rmat: n = 2^scale, llround(n * edge_factor) samples; quadrant
 * thresholds lround(p * 65536) over 16-bit draws; weights (unless w_lo == w_hi == 1) uniform in
 * [w_lo, w_hi) from the undirected pair's hash, lo + (hi - lo) * (24 random bits / 2^24), the
 * product rounded before the sum. Returns 0, 1 for bad arguments, 3 when memory runs out. */
int og_gen_rmat(int scale, double edge_factor, double a, double b, double c, uint64_t seed, float w_lo,
                float w_hi, int threads, og_graph *out) {
  if (!out || scale < 1 || scale > 31 || !(edge_factor > 0) || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 ||
      w_hi < w_lo)
    return 1;
  memset(out, 0, sizeof(*out));
  set_threads(threads);
  const int64_t n = (int64_t)1 << scale;
  gen g;
  memset(&g, 0, sizeof(g));
  g.kind = 0;
  g.scale = scale;
  g.krmat = stream_key(seed, STREAM_RMAT);
  g.tA = (uint32_t)lround(a * 65536.0);
  g.tAB = (uint32_t)lround((a + b) * 65536.0);
  g.tABC = (uint32_t)lround((a + b + c) * 65536.0);
  if (build_symmetric(&g, n, (int64_t)llround((double)n * edge_factor), out) != 0) return 3;
  if (!(w_lo == 1.0f && w_hi == 1.0f)) {
    out->wt = (float *)malloc((size_t)(out->m > 0 ? out->m : 1) * 4);
    if (!out->wt) { og_free(out); return 3; }
    const uint64_t kw = stream_key(seed, STREAM_WEIGHT);
    const float span = w_hi - w_lo;
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t u = 0; u < n; ++u)
      for (int64_t e = out->off[u]; e < out->off[u + 1]; ++e) {
        const uint64_t x = (uint64_t)u, y = out->tgt[e];
        const uint64_t key = x < y ? (x << 32 | y) : (y << 32 | x);
        const float t = span * ((float)(mix64(kw + key) >> 40) * (1.0f / 16777216.0f));
        out->wt[e] = w_lo + t;
      }
  }
  return 0;
}

/* The library's rak_gen_lattice: width x height 4-neighbour grid, each undirected edge deleted
 * with probability p_delete (24-bit draw below lround(p * 2^24)), plus llround(edges *
 * shortcut_frac) uniform random shortcuts; unit weights. Returns 0, 1 for bad arguments, 3 when
 * memory runs out. */
int og_gen_lattice(int64_t width, int64_t height, double p_delete, double shortcut_frac, uint64_t seed,
                   int threads, og_graph *out) {
  if (!out || width < 1 || height < 1 || width * height >= ((int64_t)1 << 31) || p_delete < 0 || p_delete > 1 ||
      shortcut_frac < 0)
    return 1;
  memset(out, 0, sizeof(*out));
  set_threads(threads);
  gen g;
  memset(&g, 0, sizeof(g));
  g.kind = 1;
  g.width = width;
  g.n = width * height;
  g.eh = (width - 1) * height;
  g.grid = g.eh + width * (height - 1);
  g.del24 = (uint32_t)lround(p_delete * 16777216.0);
  g.klat = stream_key(seed, STREAM_LATTICE);
  g.klat2 = stream_key(seed, STREAM_LATTICE + 16);
  const int64_t shortcuts = (int64_t)llround((double)g.grid * shortcut_frac);
  return build_symmetric(&g, g.n, g.grid + shortcuts, out) != 0 ? 3 : 0;
}
