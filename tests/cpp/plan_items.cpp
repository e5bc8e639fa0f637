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
  std::printf("ok\n");
  return 0;
}
