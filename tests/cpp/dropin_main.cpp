// A reference-style caller of the C++ drop-in (include/rak_lowmem.hpp): a graph type with the
// reference's interface and ids 1..n (vertex 0 absent, as the reference's MTX reader makes them),
// two 5-cliques joined by a bridge, run through rakLowmemStaticCuda<8> and <1>.
#include <cstdio>
#include <utility>
#include <vector>

#include "rak_lowmem.hpp"

struct ToyGraph {
  using key_type = uint32_t;
  using edge_value_type = float;
  std::vector<std::vector<std::pair<uint32_t, float>>> adj;  // index = vertex id, 0 unused
  size_t span() const { return adj.size(); }
  size_t order() const { return adj.size() - 1; }
  template <class F> void forEachVertexKey(F f) const { for (uint32_t u = 1; u < adj.size(); ++u) f(u); }
  template <class F> void forEachEdge(uint32_t u, F f) const { for (auto &e : adj[u]) f(e.first, e.second); }
  void addEdge(uint32_t u, uint32_t v) { adj[u].push_back({v, 1.0f}); adj[v].push_back({u, 1.0f}); }
};

int main() {
  ToyGraph x;
  x.adj.resize(11);
  for (uint32_t b : {1u, 6u})
    for (uint32_t i = b; i < b + 5; ++i)
      for (uint32_t j = i + 1; j < b + 5; ++j) x.addEdge(i, j);
  x.addEdge(5, 6);
  try {
    auto a = rak_b200::rakLowmemStaticCuda<8>(x, {1});
    auto b = rak_b200::rakLowmemStaticCuda<1>(x, {1, 0.05, 20});
    rak_options sync;
    rak_options_default(&sync);
    sync.mode = RAK_MODE_SYNC;  // deterministic: checked against the oracle by the test
    auto c = rak_b200::rakLowmemCuda<ToyGraph, uint32_t>(x, nullptr, {1}, 8, &sync);
    for (auto *r : {&a.membership, &b.membership, &c.membership}) {
      for (size_t u = 0; u < r->size(); ++u) printf("%u ", unsigned((*r)[u]));
      printf("\n");
    }
    printf("iterations %d %d time %.3f memory %.6f\n", a.iterations, b.iterations, a.time, a.memory);
    return 0;
  } catch (const rak_b200::Error &e) {
    printf("error %d %s\n", int(e.status), e.what());
    return 3;
  }
}
