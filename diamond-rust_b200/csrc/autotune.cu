// The autotuner of the batched search: picks the context's tile and routing
// choices (drg_tuning) for a workload by timing whole searches of it.
//
// Every choice only moves work between kernels or reshapes tiles, so results
// are the same under each; what changes is the device time of a search
// (drg_run_stats.ms_total, CUDA events).  The search runs once untimed and
// then `reps` times per candidate, and the median counts.  Coordinate descent
// over the lists of include/drgpu.h, starting from the context's tuning: a
// value is kept when it is at least 1 % faster.  The best tuning is stored in
// a cache file under a key of the device, the preset and the workload's size
// (powers of two of its query and database letters), so later runs on that
// kind of workload skip the timing.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "context.h"
#include "kernels.h"

using namespace drg;

namespace {

int log2_ceil(uint64_t x) {
  int b = 0;
  while ((1ull << b) < x && b < 63) ++b;
  return b;
}

std::string cache_key(drg_ctx* c, const drg_db* db, const drg_batch* b, const drg_search_config* cfg) {
  cudaDeviceProp prop{};
  DRG_CUDA(cudaGetDeviceProperties(&prop, c->device));
  std::string name = prop.name;
  for (char& ch : name)
    if (ch == ' ') ch = '_';
  std::ostringstream k;
  k << name << "|" << (cfg->sensitivity ? cfg->sensitivity : "default") << "|q" << log2_ceil(b->total + 1) << "|d"
    << log2_ceil(db->total + 1);
  return k.str();
}

bool read_cache(const char* path, const std::string& key, drg_tuning* out) {
  if (!path) return false;
  std::ifstream f(path);
  std::string line;
  bool found = false;
  while (std::getline(f, line)) {  // the last line of a key wins
    std::istringstream in(line);
    std::string k;
    drg_tuning t{};
    if (in >> k >> t.sw_wide_min_width >> t.sw_min_packed_width >> t.sw_transpose >> t.sort_small_tiles && k == key) {
      *out = t;
      found = true;
    }
  }
  return found;
}

double time_search(drg_ctx* c, const drg_db* db, const drg_batch* b, const drg_search_config* cfg, int reps) {
  std::vector<double> ms;
  for (int r = 0; r <= reps; ++r) {
    drg_result res;
    search(c, db, b, cfg, &res);
    const double t = res.stats.ms_total;
    drg_result_free(&res);
    if (r > 0) ms.push_back(t);  // the first search is untimed
  }
  std::sort(ms.begin(), ms.end());
  return ms[ms.size() / 2];
}

}  // namespace

extern "C" int drg_autotune(drg_ctx* c, const drg_db* db, const drg_batch* b, const drg_search_config* cfg,
                            const char* cache_path, int32_t reps, drg_tuning* out, double* ms_default,
                            double* ms_best) {
  if (!c || !db || !b || !cfg || reps < 1) return DRG_ERR_INVALID;
  try {
    DRG_CUDA(cudaSetDevice(c->device));
    const std::string key = cache_key(c, db, b, cfg);
    drg_tuning t;
    if (read_cache(cache_path, key, &t)) {
      const int rc = drg_ctx_set_tuning(c, &t);
      if (rc != DRG_OK) return rc;
      if (out) *out = t;
      if (ms_default) *ms_default = 0;
      if (ms_best) *ms_best = 0;
      return DRG_OK;
    }
    drg_tuning best = c->tuning;
    double t_best = time_search(c, db, b, cfg, reps);
    if (ms_default) *ms_default = t_best;
    // the knobs in the order tuned, each with its list of values
    const std::vector<std::vector<int32_t>> lists = {{273, 137, 545, 1701}, {17, 33}, {1, 0}, {0, 1}};
    auto knob = [](drg_tuning& x, size_t k) -> int32_t& {
      return k == 0 ? x.sw_wide_min_width : k == 1 ? x.sw_min_packed_width : k == 2 ? x.sw_transpose
                                                                                     : x.sort_small_tiles;
    };
    for (size_t k = 0; k < lists.size(); ++k) {
      for (int32_t v : lists[k]) {
        if (knob(best, k) == v) continue;
        drg_tuning trial = best;
        knob(trial, k) = v;
        c->tuning = trial;
        const double ms = time_search(c, db, b, cfg, reps);
        if (ms < 0.99 * t_best) {
          t_best = ms;
          best = trial;
        }
      }
    }
    c->tuning = best;
    if (ms_best) *ms_best = t_best;
    if (out) *out = best;
    if (cache_path) {
      std::ofstream f(cache_path, std::ios::app);
      f << key << " " << best.sw_wide_min_width << " " << best.sw_min_packed_width << " " << best.sw_transpose << " "
        << best.sort_small_tiles << "\n";
    }
    return DRG_OK;
  } catch (const Error& e) {
    c->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    c->err = e.what();
    return DRG_ERR_INVALID;
  }
}
