// Host thread pool of the search's CPU-side steps: every index is visited
// exactly once, for many sizes, grains and part limits, call after call.
#include <atomic>
#include <cstdio>
#include <vector>

#include "host/pool.h"

int main() {
  for (unsigned workers : {0u, 1u, 3u, 15u}) {
    drg::host::Pool pool(workers);
    for (int rep = 0; rep < 200; ++rep) {
      const uint64_t n = (uint64_t)(rep * 37 % 5000);
      std::vector<std::atomic<int>> hit(n);
      for (auto& h : hit) h = 0;
      const uint64_t grain = 1 + rep % 300, max_parts = rep % 5;
      pool.parallel_for(n, grain, max_parts, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; ++i) hit[i]++;
      });
      for (uint64_t i = 0; i < n; ++i)
        if (hit[i] != 1) {
          std::printf("workers %u rep %d: index %llu visited %d times\n", workers, rep, (unsigned long long)i,
                      (int)hit[i]);
          return 1;
        }
    }
  }
  std::printf("ok\n");
  return 0;
}
