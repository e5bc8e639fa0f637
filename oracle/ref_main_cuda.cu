// ref_main_cuda.cu -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own GPU path, rakLowmemStaticCuda<SLOTS> (inc/rakLowmemCuda.hxx:624-632),
// on a CSR read from a file, as a separate process (the reference exits the process on any CUDA
// error, inc/_cuda.hxx:221-235, and sets device flags on every call, inc/rakLowmemCuda.hxx:570).
// Built by oracle/Makefile into oracle/_ref/ref_lpa_cuda from the reference headers in place.
//
// usage: ref_lpa_cuda <graph.rakcsr> <slots: 1|8|0> <labels.out> [repeat] [tolerance] [max_iter]
// (slots 0 runs the reference's ν-LPA, rakStaticCuda, inc/rakCuda.hxx:438-446, for comparison).
// File format (written by tests and bench): "RAKCSR01", int64 n, int64 m, int32 has_weights,
// int64 offsets[n+1], uint32 targets[m], float weights[m] (if has_weights).
// Prints one JSON line: iterations, time_ms, marking/initialization ms, memory_gb.
#define BUILD 0
#define OPENMP 1
#define CUDA 1
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <omp.h>
#include "_main.hxx"
#include "csr.hxx"
#include "properties.hxx"
#include "hashtableCuda.hxx"
#include "sketchCuda.hxx"
#include "rak.hxx"
#include "rakCuda.hxx"
#include "rakLowmemCuda.hxx"

using std::vector;

struct ShiftedCsr {
  using key_type = uint32_t;
  using vertex_value_type = None;
  using edge_value_type = float;
  int64_t n;
  const int64_t *off;
  const uint32_t *tgt;
  const float *wt;
  size_t span() const noexcept { return size_t(n) + 1; }
  size_t order() const noexcept { return size_t(n); }
  size_t size() const noexcept { return size_t(off[n]); }
  bool hasVertex(uint32_t u) const noexcept { return u >= 1 && int64_t(u) <= n; }
  size_t degree(uint32_t u) const noexcept { return hasVertex(u) ? size_t(off[u] - off[u - 1]) : 0; }
  template <class F> void forEachVertexKey(F f) const noexcept {
    for (int64_t u = 1; u <= n; ++u) f(uint32_t(u));
  }
  template <class F> void forEachEdge(uint32_t u, F f) const noexcept {
    if (!hasVertex(u)) return;
    for (int64_t i = off[u - 1]; i < off[u]; ++i) f(uint32_t(tgt[i] + 1), wt ? wt[i] : 1.0f);
  }
  template <class F> void forEachEdgeKey(uint32_t u, F f) const noexcept {
    if (!hasVertex(u)) return;
    for (int64_t i = off[u - 1]; i < off[u]; ++i) f(uint32_t(tgt[i] + 1));
  }
};

int main(int argc, char **argv) {
  if (argc < 4) { fprintf(stderr, "usage: %s graph slots labels [repeat] [tol] [maxit]\n", argv[0]); return 2; }
  FILE *f = fopen(argv[1], "rb");
  if (!f) { perror("open"); return 2; }
  char magic[8]; int64_t n, m; int32_t hw;
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "RAKCSR01", 8) || fread(&n, 8, 1, f) != 1 ||
      fread(&m, 8, 1, f) != 1 || fread(&hw, 4, 1, f) != 1) { fprintf(stderr, "bad header\n"); return 2; }
  vector<int64_t> off(n + 1); vector<uint32_t> tgt(m); vector<float> wt(hw ? m : 0);
  if (fread(off.data(), 8, n + 1, f) != size_t(n + 1) || fread(tgt.data(), 4, m, f) != size_t(m) ||
      (hw && fread(wt.data(), 4, m, f) != size_t(m))) { fprintf(stderr, "short file\n"); return 2; }
  fclose(f);
  int slots = atoi(argv[2]);
  int repeat = argc > 4 ? atoi(argv[4]) : 1;
  double tol = argc > 5 ? atof(argv[5]) : 0.05;
  int maxit = argc > 6 ? atoi(argv[6]) : 20;
  ShiftedCsr x{n, off.data(), tgt.data(), hw ? wt.data() : nullptr};
  RakOptions o(repeat, tol, maxit);
  vector<uint32_t> labels(n);
  int iters = 0; float tms = 0, tmark = 0, tinit = 0, mem = 0;
  auto take = [&](auto &r) {
    for (int64_t u = 0; u < n; ++u) labels[u] = r.membership[u + 1];
    iters = r.iterations; tms = r.time; tmark = r.markingTime; tinit = r.initializationTime; mem = r.memory;
  };
  if (slots == 1) { auto r = rakLowmemStaticCuda<1>(x, o); take(r); }
  else if (slots == 8) { auto r = rakLowmemStaticCuda<8>(x, o); take(r); }
  else if (slots == 0) { auto r = rakStaticCuda(x, o); take(r); }  // ν-LPA (hashtable per vertex)
  else { fprintf(stderr, "slots must be 0 (nu-LPA), 1 or 8\n"); return 2; }
  FILE *g = fopen(argv[3], "wb");
  if (!g || fwrite(labels.data(), 4, n, g) != size_t(n)) { perror("write"); return 2; }
  fclose(g);
  printf("{\"iterations\": %d, \"time_ms\": %.4f, \"marking_ms\": %.4f, \"init_ms\": %.4f, \"memory_gb\": %.6f}\n",
         iters, tms, tmark, tinit, mem);
  return 0;
}
