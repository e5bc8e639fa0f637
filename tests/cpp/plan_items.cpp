// Host check of the one-lane work-item arithmetic (rak_internal.hpp): for many region sizes and
// grid sizes, the items of region 6 (region_items with lane_item_for's choice) and the kernel's
// loop over them (item `local` covers batches local*lane_item + sb, sb < lane_item, stopping at the
// first batch past the region; each batch covers 32 vertices) visit every one-lane vertex exactly
// once. Prints "ok" or the first failing case.
#include <cstdio>
#include <vector>

#include "rak_internal.hpp"

int main() {
  const long long warps_list[] = {1, 24, 3552, 1776, 100000};
  for (long long cnt = 0; cnt < 20000; cnt += (cnt < 2000 ? 1 : 97)) {
    for (long long warps : warps_list) {
      const int64_t li = rak::lane_item_for(cnt, warps);
      if (li < 1 || li > 4) { std::printf("lane_item %lld for %lld\n", (long long)li, cnt); return 1; }
      const int64_t items = rak::region_items(rak::REG_LANE, cnt, 0, li);
      std::vector<int> seen(size_t(cnt), 0);
      for (int64_t local = 0; local < items; ++local)
        for (int64_t sb = 0; sb < li; ++sb) {
          const int64_t sub = local * li + sb;
          if (sub * 32 >= cnt) break;
          for (int64_t lane = 0; lane < 32; ++lane) {
            const int64_t idx = sub * 32 + lane;
            if (idx < cnt) ++seen[size_t(idx)];
          }
        }
      for (long long v = 0; v < cnt; ++v)
        if (seen[size_t(v)] != 1) {
          std::printf("vertex %lld seen %d times (cnt %lld, warps %lld, lane_item %lld)\n", v, seen[size_t(v)], cnt,
                      warps, (long long)li);
          return 1;
        }
      if (items > 0 && (items - 1) * li * 32 >= cnt) { std::printf("spare item (cnt %lld)\n", cnt); return 1; }
    }
  }
  // the thresholds: 4 batches per item only when every warp still gets 8 or more items
  if (rak::lane_item_for(32LL * 32 * 3552, 3552) != 4 || rak::lane_item_for(32LL * 16 * 3552, 3552) != 2 ||
      rak::lane_item_for(32LL * 16 * 3552 - 32, 3552) != 1) {
    std::printf("thresholds\n");
    return 1;
  }
  // plan keys: every degree maps into the histogram's range and to its region -- one lane up to
  // lane_max, split vertices above hub_min, else the smallest group G >= 2 (power of two, <= 32)
  // with G * lane_max >= degree
  const rak::Layout layouts[] = {{256, 65536, 8192}, {8, 64, 32}, {128, 8192, 4096}, {1, 1, 32}, {32, 4096, 2048}};
  for (const rak::Layout &ly : layouts) {
    const int64_t nkeys = 6 + ly.lane_max + 1;
    for (int64_t deg = 0; deg <= 2 * ly.hub_min + 10; ++deg) {
      const uint32_t k = rak::plan_key(deg, ly);
      const int r = rak::key_region(k);
      bool ok = int64_t(k) < nkeys;
      if (deg == 0) ok = ok && int64_t(k) == nkeys - 1;
      else if (deg <= ly.lane_max) ok = ok && r == rak::REG_LANE;
      else if (deg > ly.hub_min) ok = ok && r == rak::REG_HUB;
      else {
        const int64_t G = rak::region_group(r);
        ok = ok && r >= 1 && r <= 5 && (G * ly.lane_max >= deg || G == 32) && (G == 2 || (G / 2) * ly.lane_max < deg);
      }
      if (!ok) {
        std::printf("plan_key(%lld) = %u, region %d (layout %lld/%lld)\n", (long long)deg, k, r,
                    (long long)ly.lane_max, (long long)ly.hub_min);
        return 1;
      }
    }
  }
  std::printf("ok\n");
  return 0;
}
