// search::run (search.rs:95-146) on one GPU.
//
// Device stages per index chunk (seed.rs:146-164 chunking, search.rs:127-133):
//   seeds   query seeds once, reference seeds per chunk: enumerate + radix sort
//   join    query key runs x sorted reference keys, expansion cap, packed hits
//   hits    radix sort by (target, subject, diagonal, spos), de-duplicate
//   xdrop   one thread per (target, subject, diagonal) run, cutoff 19
//   bands   one thread per pair: merge, order, window (search.rs:206-230, 303-312)
//   sw      packed 16-bit banded SW scores (warp = 32 bands of one query)
//   gate    ALP E-value and the max_hsps band walk per pair
// Host: exact E-values of the kept bands, per-target culling (search.rs:256-270),
// then the exact traceback kernel for the surviving HSPs only.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <thread>
#include <cmath>
#include <cstring>
#include <numeric>

#include "context.h"
#include "kernels.h"

namespace drg {

namespace {

constexpr double kLn2 = 0.693147180559945309417232121458176568;

template <typename F>
void cub_call(drg_ctx* c, F f) {
  size_t bytes = 0;
  DRG_CUDA(f(nullptr, bytes));
  void* t = c->cub_tmp.ensure(bytes);
  DRG_CUDA(f(t, bytes));
}

// The library's radix sort on the context's stream (no host wait).
template <typename K>
SortResult<K> dsort(drg_ctx* c, K* k, K* k_alt, uint32_t* v, uint32_t* v_alt, uint64_t n, int begin_bit,
                    int end_bit, const uint64_t* d_n = nullptr) {
  return radix_sort<K>(k, k_alt, v, v_alt, n, d_n, begin_bit, end_bit, c->sort_tmp, c->sort_err.as<uint32_t>(1),
                       c->stream, c->tuning.sort_small_tiles != 0);
}

template <typename T>
T fetch(drg_ctx* c, const T* d) {
  T* h = c->h_stage.as<T>(1);
  DRG_CUDA(cudaMemcpyAsync(h, d, sizeof(T), cudaMemcpyDeviceToHost, c->stream));
  DRG_CUDA(cudaStreamSynchronize(c->stream));
  return *h;
}

template <typename T>
void fetch_n(drg_ctx* c, std::vector<T>& out, const T* d, size_t n) {
  out.resize(n);
  if (n == 0) return;
  DRG_CUDA(cudaMemcpyAsync(out.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, c->stream));
  DRG_CUDA(cudaStreamSynchronize(c->stream));
}

// Indices i < n with flags[i] != 0, in order; their count goes to the
// device word d_count (no wait).
void select_indices_dev(drg_ctx* c, const uint8_t* flags, uint64_t n, uint32_t* out, int64_t* d_count) {
  if (n == 0) return;
  thrust::counting_iterator<uint32_t> it(0);
  cub_call(c, [&](void* t, size_t& b) {
    return cub::DeviceSelect::Flagged(t, b, it, flags, out, d_count, (int64_t)n, c->stream);
  });
}

// Indices i < n with flags[i] != 0, in order.
uint64_t select_indices(drg_ctx* c, const uint8_t* flags, uint64_t n, uint32_t* out, int64_t* d_count) {
  if (n == 0) return 0;
  thrust::counting_iterator<uint32_t> it(0);
  cub_call(c, [&](void* t, size_t& b) {
    return cub::DeviceSelect::Flagged(t, b, it, flags, out, d_count, (int64_t)n, c->stream);
  });
  return (uint64_t)fetch(c, d_count);
}

// Device time of a stage on the context's stream, added to a stats field
// when the search's TimeLog resolves (no wait here).
struct Timer {
  drg_ctx* c;
  TimeLog* log;
  cudaEvent_t a = nullptr;
  Timer(drg_ctx* ctx, TimeLog* times) : c(ctx), log(times) {}
  void start() {
    a = log->event();
    DRG_CUDA(cudaEventRecord(a, c->stream));
  }
  void stop(double* dst) {
    cudaEvent_t b = log->event();
    DRG_CUDA(cudaEventRecord(b, c->stream));
    log->span(a, b, dst);
  }
};

template <typename K>
__global__ void k_count_valid(const K* keys, uint64_t n, int64_t* out) {
  // number of keys before the first "no seed" (all ones; keys sorted ascending)
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    uint64_t m = (lo + hi) >> 1;
    if (keys[m] < (K)kNoSeed) lo = m + 1;
    else hi = m;
  }
  *out = (int64_t)lo;
}

template <typename K>
int64_t count_valid(drg_ctx* c, const K* keys, uint64_t n, int64_t* d_tmp) {
  if (n == 0) return 0;
  count_launch();
  k_count_valid<K><<<1, 1, 0, c->stream>>>(keys, n, d_tmp);
  DRG_CUDA(cudaGetLastError());
  return fetch(c, d_tmp);
}

__global__ void k_set_u64(uint64_t* p, uint64_t v) { *p = v; }
__global__ void k_add_u64(unsigned long long* p, const unsigned long long* v) { *p += *v; }

// flags of each pair's first band, over a bound n of the device count *d_n
// (0 past the count)
__global__ void k_rank0_flags_dev(const Band* b, uint64_t n, const int64_t* d_n, uint8_t* f) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) f[i] = i < (uint64_t)*d_n && b[i].rank == 0;
}
// p[*at] = *v (an index array's end marker at a device-side count)
__global__ void k_set_at(uint32_t* p, const int64_t* at, const int64_t* v) { p[*at] = (uint32_t)*v; }

__host__ __device__ __forceinline__ int sw_class_of(uint32_t w) {
  return w <= (uint32_t)kSwC0 ? 0 : (w <= (uint32_t)kSwC1 ? 1 : (w <= (uint32_t)kSwC2 ? 2 : 3));
}

// Score-pass sort key, radix-sorted over bits kKeyLo..end:
//   end - 1 wide band (one warp per band, after every packed-kernel band),
//   end - 2 transposed band, 24..end - 3 group (target << 16 | window start,
//   or the subject of a transposed band), 13..23 width.  Not computed: ~0.
// (Medium bands share warps with the narrow bands of their group: giving
// them warps of their own left most of those warps' lanes idle.)
// The two flags sit right above the group field, whose width the batch sets
// (SwKeyBits), so the sort covers only the bits the keys use.
struct SwKeyBits {
  uint64_t transposed, wide;  // flag bits
  int end;                    // bits [kKeyLo, end) are sorted
};
// Task and band-job sort keys: class or route (< 8) above a cost field whose
// inverse orders longest first; the order only schedules, so costs saturate.
constexpr int kCostBits = 21;  // 2M column steps: above any warp but the rarest, so the keys sort in 3 passes
constexpr uint64_t kCostMax = (1ull << kCostBits) - 1;
constexpr int kGroupShift = 24, kWidthShift = 13, kKeyLo = 13;

// DP rows [rs, re] of a band with at least one in-matrix cell: rows are the
// query window (d = i - j in [d0, d1]) or, transposed, the subject (the
// diagonals become [-d1, -d0] and the columns are the query window).
__host__ __device__ __forceinline__ void band_rows(const Band& b, int64_t m, bool transposed, int64_t* rs,
                                                   int64_t* re) {
  const int64_t n = b.n;
  if (!transposed) {
    *rs = b.d0 + 1 > 1 ? b.d0 + 1 : 1;
    *re = m + b.d1 < n ? m + b.d1 : n;
  } else {
    *rs = -(int64_t)b.d1 + 1 > 1 ? -(int64_t)b.d1 + 1 : 1;
    *re = n - b.d0 < m ? n - b.d0 : m;
  }
}

// Number of sorted keys below `bound`.
// After a run-length encoding of n sorted seed keys into io[0] runs (keys
// rk): io[0] = runs of valid keys (the last run is dropped when it is the
// "no seed" run), io[1] = valid keys.
template <typename K>
__global__ void k_valid_runs(const K* keys, uint64_t n, const K* rk, int64_t* io) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t m = (lo + hi) >> 1;
    if (keys[m] < (K)kNoSeed) lo = m + 1;
    else hi = m;
  }
  const int64_t runs = io[0];
  io[0] = runs > 0 && rk[runs - 1] == (K)kNoSeed ? runs - 1 : runs;
  io[1] = (int64_t)lo;
}
__global__ void k_widen_keys(const uint32_t* in, uint64_t n, uint64_t* out) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

// Sorted band keys: out[0] = keys below kNoSeed (bands the packed kernels
// take), out[1] = keys below the wide flag (narrow bands, which sort first).
__global__ void k_count_fast_narrow(const uint64_t* keys, uint64_t n, uint64_t wide_key, int64_t* out) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t m = (lo + hi) >> 1;
    if (keys[m] < kNoSeed) lo = m + 1;
    else hi = m;
  }
  out[0] = (int64_t)lo;
  hi = lo;
  lo = 0;
  while (lo < hi) {
    const uint64_t m = (lo + hi) >> 1;
    if (keys[m] < wide_key) lo = m + 1;
    else hi = m;
  }
  out[1] = (int64_t)lo;
}

// The tuned routing (drg_tuning): where the packed 16-bit kernel starts, where
// the score pass hands bands to the band kernel, and whether it transposes.
struct SwTune {
  int wide_min, min_packed, transpose;
};
SwTune sw_tune(const drg_ctx* c, const Scoring& scr) {
  SwTune t{c->tuning.sw_wide_min_width, c->tuning.sw_min_packed_width, c->tuning.sw_transpose};
  if (scr.gap_open + scr.gap_extend > kSwMaxOpenCost) t.wide_min = t.min_packed;  // no packed-kernel bands
  return t;
}

// Which kernel a band goes to: the packed kernel (fast), its wide-band
// variant (wide), and whether the band has fewer strips transposed.
struct SwRoute {
  bool fast, wide, tr;
  int64_t rs, re, ts, te;
};
__device__ __forceinline__ SwRoute sw_route(const Band& b, const uint64_t* s_offsets, int max_score,
                                            const SwTune& tn) {
  SwRoute r;
  const int64_t W = (int64_t)b.d1 - b.d0 + 1;
  const int64_t m = (int64_t)(s_offsets[b.subject + 1] - s_offsets[b.subject]);
  band_rows(b, m, false, &r.rs, &r.re);
  band_rows(b, m, true, &r.ts, &r.te);
  const int64_t mn = m < (int64_t)b.n ? m : (int64_t)b.n;
  r.fast = W >= tn.min_packed && W <= kSwMaxWidth && (int64_t)max_score * mn <= kSwPackedMaxBest && r.rs <= r.re &&
           b.target < (1u << 21) && b.q0 < 65536 && r.re < 65536;
  r.wide = r.fast && W >= tn.wide_min;
  // narrow bands only: a medium band (W > 136) in a subject's warps would
  // make its narrow lanes wait on its width
  r.tr = tn.transpose && r.fast && !r.wide && W <= kSwC0 && r.ts <= r.te && r.te < 65536 &&
         (r.te - r.ts + 16) / 16 < (r.re - r.rs + 16) / 16;
  return r;
}
// Bands per subject that would run with fewer strips transposed; each such
// band draws a ticket (its arrival order, which varies from run to run: the
// grouping of bands into warps does not change any score).
__global__ void k_sw_tr_count(const Band* bands, uint64_t n, const uint64_t* s_offsets, int max_score, SwTune tn,
                              uint32_t* count, uint32_t* ticket) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Band b = bands[i];
  ticket[i] = sw_route(b, s_offsets, max_score, tn).tr ? atomicAdd(count + b.subject, 1u) : 0xFFFFFFFFu;
}

// The two sort keys of the score pass: the key above, and rows (first-row
// strip bucket, last row, the last row descending in odd buckets).  Bands are
// sorted by rows, then stably by key, so that bands next to each other cover
// nearly the same rows.
// rows[i] holds band i's ticket from k_sw_tr_count on entry.
__global__ void k_sw_keys(const Band* bands, uint64_t n, const uint64_t* s_offsets, int max_score, SwTune tn,
                          SwKeyBits kb, const uint32_t* tr_count, uint64_t* keys, uint32_t* rows, uint32_t* order) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Band b = bands[i];
  const uint64_t W = (uint64_t)(b.d1 - b.d0 + 1);
  const SwRoute r = sw_route(b, s_offsets, max_score, tn);
  // A subject's transposed bands form warps of their own: only whole warps
  // of them are transposed, the rest stay with their query windows.
  const bool tr = r.tr && tr_count && rows[i] < (tr_count[b.subject] & ~31u);
  const int64_t rs = tr ? r.ts : r.rs, re = tr ? r.te : r.re;
  const uint64_t group = tr ? (kb.transposed | ((uint64_t)b.subject << kGroupShift))
                            : ((((uint64_t)b.target << 16) | b.q0) << kGroupShift);
  keys[i] = !r.fast ? ~0ull
                    : r.wide ? (kb.wide | (W << kWidthShift))
                             : (group | (W << kWidthShift));
  const uint32_t bucket = r.fast ? (uint32_t)(rs >> 4) : 0xFFFFu;
  const uint32_t last = r.fast ? (uint32_t)re : 0u;
  rows[i] = (bucket << 16) | ((bucket & 1) ? 0xFFFFu - last : last);
  order[i] = (uint32_t)i;
}
__global__ void k_gather_keys(const uint64_t* keys, const uint32_t* idx, uint64_t n, uint64_t* out) {
  uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k < n) out[k] = keys[idx[k]];
}
__device__ __forceinline__ int64_t band_first_row(const Band& b) { return b.d0 + 1 > 1 ? b.d0 + 1 : 1; }

// Task heads: first band of each (target, window) group and every 32nd after
// (a group's bands are in width order, so a warp's widths are close).
// (d_n: the count is *d_n, n bounds it)
__global__ void k_sw_group_start(const uint64_t* keys, uint64_t n, uint32_t* gstart, const int64_t* d_n) {
  uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (s >= n || (d_n && s >= (uint64_t)*d_n)) return;
  gstart[s] = (s == 0 || (keys[s] >> kGroupShift) != (keys[s - 1] >> kGroupShift)) ? (uint32_t)s : 0u;
}
__global__ void k_sw_task_flags(const uint32_t* gstart, uint64_t n, uint8_t* f, const int64_t* d_n) {
  uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (s < n) f[s] = (!d_n || s < (uint64_t)*d_n) && ((s - gstart[s]) % 32) == 0;
}
__global__ void k_sw_fill_tasks(const uint32_t* starts, uint64_t n_tasks, const uint64_t* keys, uint64_t n_fast,
                                uint64_t transposed_key, const uint32_t* order, const Band* bands,
                                const uint64_t* s_offsets, bool row_limit,
                                SwTask* tasks, uint64_t* sort_key, uint32_t* sort_val, uint64_t* trace_size,
                                unsigned long long* cells_gpu, const int64_t* d_n_tasks, const int64_t* d_n_fast) {
  uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (d_n_tasks) n_tasks = (uint64_t)*d_n_tasks;
  if (d_n_fast) n_fast = (uint64_t)*d_n_fast;
  if (t >= n_tasks) return;
  uint32_t s = starts[t];
  const uint64_t grp = keys[s] >> kGroupShift;
  const bool transposed = (keys[s] & transposed_key) != 0;
  uint32_t cnt = 0;
  int64_t row_first = INT64_MAX, row_last = 0;
  uint32_t wmin = 0xFFFFFFFFu, wmax = 0;
  uint64_t lane_cells = 0;
  while (cnt < 32 && s + cnt < n_fast && (keys[s + cnt] >> kGroupShift) == grp) {
    const uint64_t key = keys[s + cnt];
    const Band b = bands[order[s + cnt]];
    int64_t m = (int64_t)(s_offsets[b.subject + 1] - s_offsets[b.subject]);
    int64_t rs, re;
    band_rows(b, m, transposed, &rs, &re);
    if (row_limit && !transposed && b.pad > 0 && (int64_t)b.pad < re) re = b.pad;  // rows up to the best
    const uint32_t w = (uint32_t)((key >> kWidthShift) & 0x7FF);
    if (re > row_last) row_last = re;
    if (rs < row_first) row_first = rs;
    if (w < wmin) wmin = w;
    if (w > wmax) wmax = w;
    lane_cells += (uint64_t)((re - rs + 16) / 16) * 16ull * (w + 16ull);
    ++cnt;
  }
  if (row_last < row_first) row_last = row_first;
  SwTask k;
  k.first = s;
  k.count = cnt;
  k.row_first = (uint32_t)row_first;
  k.n_strips = (uint32_t)((row_last - row_first + 16) / 16);
  k.width = wmax;
  k.w_min = wmin;
  k.transposed = transposed ? 1u : 0u;
  k.pad = 0;
  tasks[t] = k;
  const uint64_t steps = (uint64_t)k.n_strips * (wmax + 16ull);
  const int cls = sw_class_of(wmax);
  // class, then longest first (a scheduling order: 21 bits of steps, saturated, suffice)
  sort_key[t] = ((uint64_t)cls << kCostBits) | (kCostMax - (steps < kCostMax ? steps : kCostMax));
  sort_val[t] = (uint32_t)t;
  if (trace_size) trace_size[t] = steps * 32ull;
  if (cells_gpu) {
    atomicAdd(cells_gpu + 1, (unsigned long long)lane_cells);  // evaluated cells: counted by k_sw
    if (transposed) atomicAdd(cells_gpu + 3, (unsigned long long)cnt);
  }
}

__global__ void k_gather_tasks(const SwTask* in, const uint32_t* idx, uint64_t n, SwTask* out, const int64_t* d_n) {
  uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (t < n && (!d_n || t < (uint64_t)*d_n)) out[t] = in[idx[t]];
}

// First task of classes 1, 2 and 3 (tasks are sorted by class).
__global__ void k_task_bounds(const SwTask* tasks, uint64_t n, int64_t* out, const int64_t* d_n) {
  if (d_n) n = (uint64_t)*d_n;
  for (int c = 0; c < kSwClasses - 1; ++c) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
      uint64_t m = (lo + hi) >> 1;
      if (sw_class_of(tasks[m].width) <= c) lo = m + 1;
      else hi = m;
    }
    out[c] = (int64_t)lo;
  }
}

// Longest warp of each width class, in column steps (strips x (W + 16)).
__global__ void k_task_steps(const SwTask* tasks, uint64_t n, unsigned long long* mx, const int64_t* d_n) {
  uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (t >= n || (d_n && t >= (uint64_t)*d_n)) return;
  const SwTask k = tasks[t];
  atomicMax(mx + sw_class_of(k.width), (unsigned long long)k.n_strips * (k.width + 16ull));
}

// Ops of the traced bands, compacted in band order (each band owns n + m slots).
__global__ void k_ops_count(const ExactOut* out, uint64_t n, uint64_t* cnt) {
  uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k < n) cnt[k] = out[k].n_ops;
  else if (k == n) cnt[k] = 0;
}
__global__ void k_compact_ops(const uint32_t* ops, const uint64_t* ops_off, const ExactOut* out,
                              const uint64_t* coff, uint64_t n, uint32_t* dst) {
  uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t* src = ops + ops_off[k];
  uint32_t* o = dst + coff[k];
  for (uint32_t i = 0; i < out[k].n_ops; ++i) o[i] = src[i];
}

// Jobs of the one-warp-per-band kernel for the first n bands of the sorted
// order: rows [rs, re] (re limited to the best row when known), longest first.
// The job of sorted band k (order[k] indexes bands) and its sort key.
__device__ __forceinline__ void band_job(const uint32_t* order, uint64_t k, const Band* bands,
                                         const uint64_t* s_offsets, bool trace, SwBandJob* jobs, uint64_t* sort_key,
                                         uint32_t* sort_val, unsigned long long* max_width) {
  const uint32_t i = order[k];
  const Band b = bands[i];
  const int64_t m = (int64_t)(s_offsets[b.subject + 1] - s_offsets[b.subject]);
  int64_t re = m + b.d1 < (int64_t)b.n ? m + b.d1 : (int64_t)b.n;
  if (b.pad > 0 && (int64_t)b.pad < re) re = b.pad;  // the traceback needs no row below the best
  const int64_t rs = band_first_row(b);
  if (re < rs) re = rs;
  const uint32_t W = (uint32_t)(b.d1 - b.d0 + 1);
  SwBandJob j;
  j.band = i;
  j.row_first = (uint32_t)rs;
  j.n_strips = (uint32_t)((re - rs + 16) / 16);
  j.pad = W;
  j.trace_off = 0;
  jobs[k] = j;
  // by kernel route (sw_band_route), then longest first
  const int route = sw_band_route((int)W, trace);
  const uint64_t cost = (uint64_t)(j.n_strips - 1) * 19ull + W + 16ull;
  sort_key[k] = ((uint64_t)route << kCostBits) | (kCostMax - (cost < kCostMax ? cost : kCostMax));
  sort_val[k] = (uint32_t)k;
  atomicMax(max_width, (unsigned long long)W);
  atomicAdd(max_width + 1 + route, 1ull);
}
__global__ void k_band_jobs(const uint32_t* order, const uint64_t* keys, uint64_t n, const Band* bands,
                            const uint64_t* s_offsets, bool trace, SwBandJob* jobs, uint64_t* sort_key,
                            uint32_t* sort_val, unsigned long long* max_width) {
  uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k < n) band_job(order, k, bands, s_offsets, trace, jobs, sort_key, sort_val, max_width);
}
// Score pass on device counts: the wide bands are sorted positions
// [cnt[1], cnt[0]) (after the narrow ones); n bounds their count, which is
// also written to cnt[15] for the job sort.
__global__ void k_band_jobs_dev(const uint32_t* order, int64_t* cnt, uint64_t n, const Band* bands,
                                const uint64_t* s_offsets, SwBandJob* jobs, uint64_t* sort_key, uint32_t* sort_val,
                                unsigned long long* max_width) {
  uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t n_wide = (uint64_t)(cnt[0] - cnt[1]);
  if (k == 0) cnt[15] = (int64_t)n_wide;
  if (k < n && k < n_wide) band_job(order + cnt[1], k, bands, s_offsets, false, jobs, sort_key, sort_val, max_width);
}
__global__ void k_gather_band_jobs(const SwBandJob* in, const uint32_t* idx, uint64_t n, SwBandJob* out,
                                   uint64_t* size, const int64_t* d_n = nullptr) {
  uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (d_n) {  // device count: no sizes
    if (k < n && k < (uint64_t)*d_n) out[k] = in[idx[k]];
    return;
  }
  if (k < n) {
    const SwBandJob j = in[idx[k]];
    out[k] = j;
    size[k] = (uint64_t)j.n_strips * (j.pad + 16ull);
  } else if (k == n) {
    size[k] = 0;
  }
}
__global__ void k_set_band_trace_off(SwBandJob* jobs, const uint64_t* off, uint64_t n) {
  uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k < n) jobs[k].trace_off = off[k];
}

// Bands the packed kernel did not take, or whose best is not above the
// matrix's largest score (exact_below = that + 1): only then can a cell the
// packed kernels skip (the reference's clamped column past row m + d1) hold
// the best.
__global__ void k_exact_flags(const uint32_t* order, uint64_t n_fast, uint64_t n, const int32_t* score,
                              const TraceBand* tband, int exact_below, uint8_t* f) {
  uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t i = order[s];
  int v = tband ? tband[i].score : score[i];
  f[s] = (s >= n_fast || v < exact_below) ? 1 : 0;
}

__global__ void k_gather_positions(const uint32_t* pos, const uint32_t* order, uint64_t n, const Band* bands,
                                   uint32_t* idx, Band* out) {
  uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t i = order[pos[k]];
  idx[k] = i;
  out[k] = bands[i];
}

__global__ void k_scatter_scores(const uint32_t* idx, const ExactOut* out, uint64_t n, int32_t* score) {
  uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k < n) score[idx[k]] = out[k].score;
}

__global__ void k_scatter_exact(const uint32_t* idx, const ExactOut* src, uint64_t n, ExactOut* dst) {
  uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k < n) dst[idx[k]] = src[k];
}

__global__ void k_state_flags(const uint8_t* state, uint64_t n, uint8_t* f) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) f[i] = state[i] >= 2;
}

// (n bounds the device-side count *d_n)
__global__ void k_gather_bands_dev(const uint32_t* idx, uint64_t n, const int64_t* d_n, const Band* bands,
                                   const int32_t* score, const int32_t* best_row, const uint8_t* state, Band* out_b,
                                   int32_t* out_s, uint8_t* out_st) {
  uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= n || k >= (uint64_t)*d_n) return;
  uint32_t i = idx[k];
  Band b = bands[i];
  b.pad = best_row ? (uint32_t)best_row[i] : 0u;  // first row of the best: the traceback needs no row below
  out_b[k] = b;
  out_s[k] = score[i];
  out_st[k] = state[i];
}

}  // namespace

// The banded DP of n_bands bands (any order).  The packed kernel takes the
// bands whose width it supports (by width class) and whose best cannot
// overflow 16 bits; the exact kernel takes the rest and every band whose
// packed best is not above the matrix's largest score.
//  score mode (trace == false): scores[i] = best score (0 = None).
//  trace mode: out[i] and the band's ops at h_ops_off[i] in ops (n + m slots
//  per band), the same records the exact kernel produces.
namespace {

// Jobs of the one-warp-per-band kernel for n bands (order[k] indexes bands),
// longest first, with their trace offsets when trace is set.
struct BandJobs {
  SwBandJob* jobs = nullptr;
  uint64_t n = 0;
  int max_width = 0;
  uint64_t trace_words = 0;
  uint64_t route_lo[5] = {0, 0, 0, 0, 0};  // jobs [route_lo[r], route_lo[r + 1]) take route r
};
BandJobs make_band_jobs(drg_ctx* c, const uint32_t* order, const uint64_t* keys, uint64_t n, const Band* bc,
                        const uint64_t* s_offsets, bool trace) {
  BandJobs r;
  r.n = n;
  if (n == 0) return r;
  SwBandJob* jobs_u = c->band_jobs_u.as<SwBandJob>(n);
  r.jobs = c->band_jobs.as<SwBandJob>(n);
  uint64_t* key = c->bj_key.as<uint64_t>(n);
  uint64_t* key_s = c->bj_key_s.as<uint64_t>(n);
  uint32_t* val = c->bj_val.as<uint32_t>(n);
  uint32_t* val_s = c->bj_val_s.as<uint32_t>(n);
  unsigned long long* dmaxw = c->bj_max.as<unsigned long long>(5);  // max width, jobs per route
  DRG_CUDA(cudaMemsetAsync(dmaxw, 0, 5 * sizeof(unsigned long long), c->stream));
  count_launch();
  k_band_jobs<<<ceil_div(n, 256), 256, 0, c->stream>>>(order, keys, n, bc, s_offsets, trace, jobs_u, key, val,
                                                       dmaxw);
  const uint32_t* val_sorted = dsort(c, key, key_s, val, val_s, n, 0, kCostBits + 3).vals;
  uint64_t* size = c->bj_size.as<uint64_t>(n + 1);
  uint64_t* off = c->bj_off.as<uint64_t>(n + 1);
  count_launch();
  k_gather_band_jobs<<<ceil_div(n + 1, 256), 256, 0, c->stream>>>(jobs_u, val_sorted, n, r.jobs, size);
  if (trace) {
    cub_call(c, [&](void* t, size_t& b) {
      return cub::DeviceScan::ExclusiveSum(t, b, size, off, (int64_t)n + 1, c->stream);
    });
    count_launch();
    k_set_band_trace_off<<<ceil_div(n, 256), 256, 0, c->stream>>>(r.jobs, off, n);
  }
  // max width, jobs per route and (trace) the trace size, in one wait
  unsigned long long* h = c->h_stage.as<unsigned long long>(6);
  DRG_CUDA(cudaMemcpyAsync(h, dmaxw, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
  if (trace) DRG_CUDA(cudaMemcpyAsync(h + 5, off + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
  DRG_CUDA(cudaStreamSynchronize(c->stream));
  r.max_width = (int)h[0];
  for (int k = 0; k < 4; ++k) r.route_lo[k + 1] = r.route_lo[k] + h[1 + k];
  if (trace) r.trace_words = h[5];
  return r;
}

// The band kernels of jobs bj, one launch per route.
void launch_band_routes(SwBandArgs ba, const BandJobs& bj, bool trace, cudaStream_t st) {
  for (int k = 0; k < 4; ++k) {
    ba.lo = bj.route_lo[k];
    ba.hi = bj.route_lo[k + 1];
    launch_sw_band_route(ba, k, bj.max_width, trace, st);
  }
}

SwBandArgs band_args(const Band* bc, const BandJobs& bj, const DevSeqs& qs, const DevSeqs& s, const Scoring& scr) {
  SwBandArgs ba{};
  ba.bands = bc;
  ba.jobs = bj.jobs;
  ba.lo = 0;
  ba.hi = bj.n;
  ba.q_letters = qs.dp_letters();
  ba.q_offsets = qs.offsets;
  ba.s_letters = s.dp_letters();
  ba.s_offsets = s.offsets;
  ba.gap_open = scr.gap_open;
  ba.gap_extend = scr.gap_extend;
  std::memcpy(ba.scores625, scr.scores, 625);
  return ba;
}

}  // namespace

void run_bands(drg_ctx* c, const Band* bc, uint64_t n_bands, const DevSeqs& qs, const DevSeqs& s,
               const Scoring& scr, bool trace, int32_t* scores, int32_t* best_row, ExactOut* out, uint32_t* ops,
               const uint64_t* d_ops_off, const std::vector<uint64_t>* h_ops_off, drg_run_stats& st,
               int64_t* d_count, unsigned long long* cells_gpu, TimeLog* times) {
  if (n_bands == 0) return;
  TimeLog own;
  TimeLog* log = times ? times : &own;
  uint8_t* flags = c->flags.as<uint8_t>(n_bands + 1);
  uint64_t* swk = c->sw_keys.as<uint64_t>(n_bands);
  uint64_t* swks = c->sw_keys_s.as<uint64_t>(n_bands);
  uint32_t* swo = c->sw_order.as<uint32_t>(n_bands);
  uint32_t* swos = c->sw_order_s.as<uint32_t>(n_bands);  // sorted keys and order: where the sorts leave them
  uint32_t* rows = c->sw_rows.as<uint32_t>(n_bands);
  uint32_t* rows_s = c->sw_rows_s.as<uint32_t>(n_bands);
  uint64_t* swk_r = c->sw_keys_r.as<uint64_t>(n_bands);
  uint32_t* swo_r = c->sw_order_r.as<uint32_t>(n_bands);
  // the score pass may transpose bands; the traceback runs them as they are
  uint32_t* tr_count = nullptr;
  if (!trace) {
    const uint64_t n_subjects = s.h_offsets->size() - 1;
    tr_count = c->tr_count.as<uint32_t>(n_subjects);
    DRG_CUDA(cudaMemsetAsync(tr_count, 0, n_subjects * sizeof(uint32_t), c->stream));
    count_launch();
    k_sw_tr_count<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(bc, n_bands, s.offsets, scr.max_score,
                                                                  sw_tune(c, scr), tr_count, rows);
  }
  count_launch();
  // group field: target << 16 | window start, or the subject (transposed)
  SwKeyBits kb;
  {
    const int gb = std::max(bits_for(qs.h_offsets->size() > 1 ? qs.h_offsets->size() - 2 : 0) + 16,
                            bits_for(s.h_offsets->size() > 1 ? s.h_offsets->size() - 2 : 0));
    kb.transposed = 1ull << (kGroupShift + gb);
    kb.wide = 1ull << (kGroupShift + gb + 1);
    kb.end = kGroupShift + gb + 2;
    if (kb.end > 64) throw Error(DRG_ERR_INVALID, "score-pass key needs more than 64 bits");
  }
  k_sw_keys<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(bc, n_bands, s.offsets, scr.max_score, sw_tune(c, scr), kb,
                                                           tr_count, swk, rows, swo);
  // rows first, then a stable sort by (target, window, width)
  uint32_t* by_rows = dsort(c, rows, rows_s, swo, swo_r, n_bands, 0, 32).vals;
  count_launch();
  k_gather_keys<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(swk, by_rows, n_bands, swk_r);
  {
    const SortResult<uint64_t> r = dsort(c, swk_r, swks, by_rows, swos, n_bands, kKeyLo, kb.end);
    swks = r.keys;
    swos = r.vals;
  }
  uint64_t n_fast = 0, n_narrow = 0;
  // score pass counts, on the device until the one wait before the launches:
  //   [0] fast bands  [1] narrow bands  [2] tasks  [3..5] class bounds
  //   [6] wide max width  [7..10] wide jobs per route  [11..14] longest warp
  //   per class  [15] wide bands
  int64_t* cnt = c->sw_counts.as<int64_t>(16);
  DRG_CUDA(cudaMemsetAsync(cnt, 0, 16 * sizeof(int64_t), c->stream));
  count_launch();
  k_count_fast_narrow<<<1, 1, 0, c->stream>>>(swks, n_bands, kb.wide, cnt);
  TraceBand* tb = nullptr;
  if (trace) {
    int64_t* h = c->h_stage.as<int64_t>(2);
    DRG_CUDA(cudaMemcpyAsync(h, cnt, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    DRG_CUDA(cudaStreamSynchronize(c->stream));
    n_fast = (uint64_t)h[0];
    n_narrow = (uint64_t)h[1];
    tb = c->tband.as<TraceBand>(n_bands);
    DRG_CUDA(cudaMemsetAsync(tb, 0xFF, n_bands * sizeof(TraceBand), c->stream));  // score -1: not traced
    if (n_fast > 0) {
      // traceback: one warp per band (few, long bands)
      const BandJobs bj = make_band_jobs(c, swos, swks, n_fast, bc, s.offsets, true);
      SwBandArgs ba = band_args(bc, bj, qs, s, scr);
      ba.trace = c->trace.as<uint2>(bj.trace_words + 8);  // the walk reads 8-word windows
      ba.tband = tb;
      cudaEvent_t e0 = log->event(), e1 = log->event();
      DRG_CUDA(cudaEventRecord(e0, c->stream));
      // each band's walk (gapped.rs:205-279) runs in the band kernel right
      // after its DP
      ba.walk.trace = ba.trace;
      ba.walk.q_letters = qs.letters;
      ba.walk.q_offsets = qs.offsets;
      ba.walk.s_letters = s.letters;
      ba.walk.s_offsets = s.offsets;
      ba.walk.ops_off = d_ops_off;
      ba.walk.rev = c->rev.as<uint8_t>((*h_ops_off)[n_bands] + 16);
      ba.walk.ops = ops;
      ba.walk.out = out;
      ba.walk.exact_below = scr.max_score + 1;
      launch_band_routes(ba, bj, true, c->stream);
      DRG_CUDA(cudaEventRecord(e1, c->stream));
      log->span(e0, e1, &st.ms_trace_kernel);
    }
  } else {
    // ---- wide bands (positions [narrow, fast) of the sorted order): band-
    // kernel jobs by route, then longest first
    SwBandJob* jobs_u = c->band_jobs_u.as<SwBandJob>(n_bands);
    SwBandJob* wjobs = c->band_jobs.as<SwBandJob>(n_bands);
    uint64_t* jkey = c->bj_key.as<uint64_t>(n_bands);
    uint64_t* jkey_s = c->bj_key_s.as<uint64_t>(n_bands);
    uint32_t* jval = c->bj_val.as<uint32_t>(n_bands);
    uint32_t* jval_s = c->bj_val_s.as<uint32_t>(n_bands);
    count_launch();
    k_band_jobs_dev<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(
        swos, cnt, n_bands, bc, s.offsets, jobs_u, jkey, jval, reinterpret_cast<unsigned long long*>(cnt + 6));
    const uint32_t* jorder =
        dsort(c, jkey, jkey_s, jval, jval_s, n_bands, 0, kCostBits + 3, reinterpret_cast<const uint64_t*>(cnt + 15))
            .vals;
    count_launch();
    k_gather_band_jobs<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(jobs_u, jorder, n_bands, wjobs, nullptr,
                                                                        cnt + 15);
    // ---- narrow bands: warps of up to 32 bands of one group
    uint32_t* gstart = c->idx.as<uint32_t>(n_bands + 1);
    count_launch();
    k_sw_group_start<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(swks, n_bands, gstart, cnt + 1);
    cub_call(c, [&](void* t, size_t& b) {
      return cub::DeviceScan::InclusiveScan(t, b, gstart, gstart, cub::Max(), (int64_t)n_bands, c->stream);
    });
    count_launch();
    k_sw_task_flags<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(gstart, n_bands, flags, cnt + 1);
    uint32_t* tstart = c->sel_idx.as<uint32_t>(n_bands + 1);
    select_indices_dev(c, flags, n_bands, tstart, cnt + 2);
    SwTask* tasks_u = c->sw_tasks_u.as<SwTask>(n_bands);
    SwTask* tasks = c->sw_tasks.as<SwTask>(n_bands);
    uint64_t* tkey = c->task_key.as<uint64_t>(n_bands);
    uint64_t* tkey_s = c->task_key_s.as<uint64_t>(n_bands);
    uint32_t* tval = c->task_val.as<uint32_t>(n_bands);
    uint32_t* tval_s = c->task_val_s.as<uint32_t>(n_bands);
    count_launch();
    k_sw_fill_tasks<<<ceil_div(n_bands, 128), 128, 0, c->stream>>>(tstart, n_bands, swks, n_bands, kb.transposed,
                                                                    swos, bc, s.offsets, false, tasks_u, tkey, tval,
                                                                    nullptr, cells_gpu, cnt + 2, cnt + 1);
    // by width class, longest warps first within a class
    const uint32_t* task_order =
        dsort(c, tkey, tkey_s, tval, tval_s, n_bands, 0, kCostBits + 2, reinterpret_cast<const uint64_t*>(cnt + 2))
            .vals;
    count_launch();
    k_gather_tasks<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(tasks_u, task_order, n_bands, tasks, cnt + 2);
    count_launch();
    k_task_bounds<<<1, 1, 0, c->stream>>>(tasks, n_bands, cnt + 3, cnt + 2);
    count_launch();
    k_task_steps<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(tasks, n_bands,
                                                                 reinterpret_cast<unsigned long long*>(cnt + 11),
                                                                 cnt + 2);
    // ---- the one wait: every count the launches need
    int64_t* h = c->h_stage.as<int64_t>(16);
    DRG_CUDA(cudaMemcpyAsync(h, cnt, 16 * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    DRG_CUDA(cudaStreamSynchronize(c->stream));
    n_fast = (uint64_t)h[0];
    n_narrow = (uint64_t)h[1];
    const uint64_t n_tasks = (uint64_t)h[2];
    int64_t bounds[kSwClasses - 1] = {h[3], h[4], h[5]};
    unsigned long long hmax[kSwClasses];
    for (int k = 0; k < kSwClasses; ++k) hmax[k] = (unsigned long long)h[11 + k];
    BandJobs wide;
    wide.jobs = wjobs;
    wide.n = n_fast - n_narrow;
    wide.max_width = (int)h[6];
    for (int k = 0; k < 4; ++k) wide.route_lo[k + 1] = wide.route_lo[k] + (uint64_t)h[7 + k];
    if (n_fast > 0) {
      SwScoreArgs sa{};
      sa.bands = bc;
      sa.order = swos;
      sa.tasks = tasks;
      sa.q_letters = qs.dp_letters();
      sa.q_offsets = qs.offsets;
      sa.s_letters = s.dp_letters();
      sa.s_offsets = s.offsets;
      sa.gap_open = scr.gap_open;
      sa.gap_extend = scr.gap_extend;
      sa.score = scores;
      sa.best_row = best_row;
      sa.cells_eval = cells_gpu;
      std::memcpy(sa.scores625, scr.scores, 625);
      uint64_t lo[kSwClasses], hi[kSwClasses];
      for (int k = 0; k < kSwClasses; ++k) {
        lo[k] = k == 0 ? 0 : (uint64_t)bounds[k - 1];
        hi[k] = k == kSwClasses - 1 ? n_tasks : (uint64_t)bounds[k];
      }
      // The bulk class runs on the main stream; the wider classes and the wide
      // bands run on the side stream, queued first so that the long warps start
      // early and the pass ends on the bulk class's shortest tasks.
      std::array<cudaEvent_t, 2 * kSwClasses + 3> ev;
      for (auto& e : ev) e = log->event();
      const int fork = 2 * kSwClasses, wide0 = fork + 1, wide1 = fork + 2;
      DRG_CUDA(cudaEventRecord(ev[fork], c->stream));
      DRG_CUDA(cudaStreamWaitEvent(c->side, ev[fork], 0));
      auto launch_cls = [&](int cls) {
        cudaStream_t sc = cls == 0 ? c->stream : c->side;
        sa.task_lo = lo[cls];
        sa.task_hi = hi[cls];
        DRG_CUDA(cudaEventRecord(ev[2 * cls], sc));
        if (hi[cls] > lo[cls]) {
          launch_sw_class(sa, cls, sc);
          st.sw_launches += 1;
        }
        DRG_CUDA(cudaEventRecord(ev[2 * cls + 1], sc));
      };
      DRG_CUDA(cudaEventRecord(ev[wide0], c->side));
      if (wide.n > 0) {
        SwBandArgs ba = band_args(bc, wide, qs, s, scr);
        ba.score = scores;
        ba.best_row = best_row;
        launch_band_routes(ba, wide, false, c->side);
        st.sw_launches += 1;
      }
      DRG_CUDA(cudaEventRecord(ev[wide1], c->side));
      for (int cls = kSwClasses - 1; cls >= 1; --cls) launch_cls(cls);
      launch_cls(0);
      const int side_end = 2 * 1 + 1;  // class 1 is the side stream's last launch
      DRG_CUDA(cudaStreamWaitEvent(c->stream, ev[side_end], 0));
      for (int k = 0; k < kSwClasses; ++k) {
        st.sw_class_tasks[k] += hi[k] - lo[k];
        if (hmax[k] > st.sw_class_max_steps[k]) st.sw_class_max_steps[k] = hmax[k];
      }
      st.sw_wide_bands += wide.n;
      drg_run_stats* stp = &st;
      log->later([ev, fork, wide0, wide1, side_end, stp] {
        float cls_ms[kSwClasses], side_span = 0, wide_ms = 0;
        for (int k = 0; k < kSwClasses; ++k) DRG_CUDA(cudaEventElapsedTime(&cls_ms[k], ev[2 * k], ev[2 * k + 1]));
        DRG_CUDA(cudaEventElapsedTime(&side_span, ev[fork], ev[side_end]));
        DRG_CUDA(cudaEventElapsedTime(&wide_ms, ev[wide0], ev[wide1]));
        stp->ms_sw_kernel += cls_ms[0] > side_span ? cls_ms[0] : side_span;  // wall of the concurrent launches
        for (int k = 0; k < kSwClasses; ++k) stp->ms_sw_class[k] += cls_ms[k];
        stp->ms_sw_wide += wide_ms;
      });
    }
  }
  // the exact kernel for the bands the packed kernel did not settle
  count_launch();
  k_exact_flags<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(swos, n_fast, n_bands, scores, tb,
                                                                scr.max_score + 1, flags);
  uint32_t* ex_pos = c->sel_idx.as<uint32_t>(n_bands + 1);
  const uint64_t n_ex = select_indices(c, flags, n_bands, ex_pos, d_count);
  st.exact_bands += n_ex;
  if (n_ex > 0) {
    uint32_t* ex_idx = c->idx.as<uint32_t>(n_ex);
    Band* ex_b = c->ex_bands.as<Band>(n_ex);
    count_launch();
    k_gather_positions<<<ceil_div(n_ex, 256), 256, 0, c->stream>>>(ex_pos, swos, n_ex, bc, ex_idx, ex_b);
    std::vector<uint32_t> bidx;
    std::vector<Band> all_b;
    fetch_n(c, bidx, ex_idx, n_ex);
    fetch_n(c, all_b, ex_b, n_ex);
    std::vector<ExactJob> jobs(n_ex);
    uint64_t soff = 0;
    for (uint64_t k = 0; k < n_ex; ++k) {
      const Band& b = all_b[k];
      ExactJob& j = jobs[k];
      j.q = qs.letters + (*qs.h_offsets)[b.target] + b.q0;
      j.s = s.letters + (*s.h_offsets)[b.subject];
      j.n = b.n;
      j.m = (uint32_t)((*s.h_offsets)[b.subject + 1] - (*s.h_offsets)[b.subject]);
      j.d0 = b.d0;
      j.d1 = b.d1;
      j.scratch_off = soff;
      j.ops_off = trace ? (*h_ops_off)[bidx[k]] : 0;
      soff += exact_scratch_bytes(j.n, j.m, j.d0, j.d1, trace);
    }
    ExactJob* dj = c->exact_jobs.as<ExactJob>(n_ex);
    ExactOut* dout = c->exact_out.as<ExactOut>(n_ex);
    uint8_t* scratch = c->exact_scratch.as<uint8_t>(soff);
    DRG_CUDA(cudaMemcpyAsync(dj, jobs.data(), n_ex * sizeof(ExactJob), cudaMemcpyHostToDevice, c->stream));
    launch_sw_exact_with_matrix(dj, n_ex, scr.gap_open, scr.gap_extend, trace, scratch, trace ? ops : nullptr, dout,
                                scr.scores, c->stream);
    count_launch();
    if (trace) k_scatter_exact<<<ceil_div(n_ex, 256), 256, 0, c->stream>>>(ex_idx, dout, n_ex, out);
    else k_scatter_scores<<<ceil_div(n_ex, 256), 256, 0, c->stream>>>(ex_idx, dout, n_ex, scores);
    DRG_CUDA(cudaGetLastError());
  }
  if (!times) {  // a call of its own: its kernel times are read now
    DRG_CUDA(cudaStreamSynchronize(c->stream));
    own.resolve();
  }
}

namespace {

struct Candidate {
  Band band;
  int32_t score;
  uint8_t state;
  uint64_t pair_key;  // chunk << 32 | pair: identifies the (target, subject) pair
  double evalue, bits;
};

struct Search {
  drg_ctx* c;
  const drg_db* db;
  const drg_batch* q;
  Scoring sc;
  std::vector<ShapeCode> shapes;
  ReducedAlphabet red;
  double complexity_cut = 0;
  int seed_key_bits = 48;  // sorted bits of a seed key (shape id and packed key)
  uint64_t index_chunks = 1;
  double evalue = 1e-3;
  uint64_t max_hsps = 1, max_targets = 25;
  uint64_t host_threads = 0;  // 0: all of the context's host threads
  uint64_t hit_budget = 1ull << 28;  // hits held before the stages after the join run
  uint64_t pass = 0;                 // passes of those stages so far
  uint64_t query_blocks = 0;         // blocks the batch was joined in (over all chunks)
  drg_run_stats st{};
  std::vector<Candidate> cands;
  // device scratch for counters
  int64_t* d_count = nullptr;
  // [0] xdrops [1] cells_ref [2] computed [3] cells_gpu [4] lane cells [5] issued cells
  // [6] transposed bands [7] valid reference seeds of chunks enumerated without an index
  unsigned long long* d_counters = nullptr;
  TimeLog times;  // stage times, read after the search's last wait

  void configure(const drg_search_config* cfg) {
    std::string err;
    if (!make_scoring(cfg->matrix ? cfg->matrix : "BLOSUM62", cfg->gap_open, cfg->gap_extend, &sc, &err))
      throw Error(DRG_ERR_INVALID, err);
    std::string sens = cfg->sensitivity ? cfg->sensitivity : "default";
    shapes = preset_shapes(sens);
    red = preset_reduction(sens);
    double cut = cfg->has_seed_cut ? cfg->seed_cut : preset_seed_cut(sens);
    complexity_cut = cut * kLn2 * (double)shapes[0].weight;
    index_chunks = cfg->index_chunks >= 0 ? std::max<int64_t>(cfg->index_chunks, 1) : preset_index_chunks(sens);
    evalue = cfg->evalue;
    max_hsps = std::max<uint32_t>(cfg->max_hsps, 1);
    max_targets = std::max<uint32_t>(cfg->max_target_seqs, 1);
    host_threads = cfg->threads;
    hit_budget = cfg->max_hits_per_pass ? cfg->max_hits_per_pass : (1ull << 28);
    if ((int)shapes.size() > kMaxShapes) throw Error(DRG_ERR_INVALID, "too many seed shapes");
    ShapeTable t{};
    t.n = (int)shapes.size();
    for (int s = 0; s < t.n; ++s) {
      if (shapes[s].weight > kMaxWeight) throw Error(DRG_ERR_INVALID, "seed shape weight above 16");
      if (shapes[s].span > kMaxSpan) throw Error(DRG_ERR_INVALID, "seed shape longer than 256 positions");
      t.weight[s] = (uint8_t)shapes[s].weight;
      t.span[s] = (uint16_t)shapes[s].span;
      for (int k = 0; k < shapes[s].weight; ++k) t.pos[s][k] = (uint8_t)shapes[s].positions[k];
    }
    SeedParams p{};
    for (int i = 0; i < 32; ++i) p.bucket[i] = 255;
    for (int i = 0; i < 25; ++i) p.bucket[i] = red.bucket[i];
    p.size = (uint64_t)red.size;
    p.cut = complexity_cut;
    ln_factorial_table(p.lnfact);
    // key layout: the widest shape key, then the shape id (one spare bit, so
    // that no valid key has all sorted bits set like "no seed"), then requests
    int kb = 0;
    for (const auto& sh : shapes) {
      uint64_t mx = 1;
      for (int k = 0; k < sh.weight; ++k) mx *= (uint64_t)red.size;
      kb = std::max(kb, bits_for(mx - 1));
    }
    p.shape_shift = kb;
    p.request_shift = kb + bits_for((uint64_t)shapes.size());
    seed_key_bits = p.request_shift;
    if (seed_key_bits + bits_for(kMaxRequests) > 64) throw Error(DRG_ERR_INVALID, "seed keys need more than 64 bits");
    upload_seed_params(t, p, c->slot, c->stream);
    upload_score_matrix(sc.scores, c->slot, c->stream);
    upload_alp_tables(c->stream);
  }

  // What the sorted reference seeds of chunk [c0, c1) depend on.
  std::string index_key(uint64_t c0, uint64_t c1) const {
    std::string k;
    for (const auto& sh : shapes) k += sh.code + ",";
    k += "|";
    for (int i = 0; i < 25; ++i) k += std::to_string((int)red.bucket[i]) + ".";
    uint64_t cut_bits;
    std::memcpy(&cut_bits, &complexity_cut, sizeof cut_bits);
    k += "|" + std::to_string(red.size) + "|" + std::to_string(cut_bits) + "|" + std::to_string(seed_key_bits) + "|" +
         std::to_string(c0) + "-" + std::to_string(c1);
    return k;
  }

  // The hit key of the current target window [t_base, t_base + t_window).
  HitKeyLayout layout() const {
    HitKeyLayout L;
    L.tb = bits_for(t_window > 0 ? t_window - 1 : 0);
    L.sb = bits_for(db->n > 0 ? db->n - 1 : 0);
    L.doff = (int64_t)db->max_len;
    L.db = bits_for((uint64_t)q->max_len + db->max_len);
    L.pb = bits_for(db->max_len);
    if (L.tb < 1) L.tb = 1;
    if (L.sb < 1) L.sb = 1;
    L.t_base = (uint32_t)t_base;
    return L;
  }
  // Targets per window: all of them when the full key fits 64 bits, else as
  // many as the bits left beside subject, diagonal and position allow (the
  // join then runs in blocks of at most that many targets).
  void set_target_window() {
    t_base = 0;
    t_window = q->n;
    const int rest = bits_for(db->n > 0 ? db->n - 1 : 0) + bits_for((uint64_t)q->max_len + db->max_len) +
                     bits_for(db->max_len);
    if (std::max(1, bits_for(q->n > 0 ? q->n - 1 : 0)) + std::max(1, rest) <= 64) return;
    if (rest > 63)
      throw Error(DRG_ERR_INVALID, "database too large: hit key needs " + std::to_string(rest + 1) + " bits");
    t_window = 1ull << (64 - rest);
  }
  uint64_t t_base = 0, t_window = 0;

  void run(drg_result* out);
  void query_seeds(uint64_t* n_runs);
  // The join of index chunk [c0, c1): its hits are appended to acc.
  void join_chunk(uint64_t c0, uint64_t c1, uint64_t n_runs);
  // bitmap of the query's seed keys (built on the first chunk that needs it)
  uint32_t* key_filter = nullptr;
  int key_filter_log2 = 0;
  void build_key_filter(uint64_t n_runs);
  // The first index chunk's reference side (key bitmap, filtered reference
  // seeds, their sort) on the side stream while the query seeds sort: no
  // index cache, no request ids, 32-bit seed keys.  The query enumeration
  // sets the bitmap; ev_qkeys: it is done; ev_ref: the chunk's sorted
  // reference seeds are ready.
  bool early_possible() const;
  void start_early_ref();
  bool early_ref = false;
  uint64_t early_c0 = 0, early_c1 = 0;
  const uint32_t* early_keys32_s = nullptr;
  const uint32_t* early_vals_s = nullptr;
  int64_t early_nr = 0;
  const uint64_t* early_d_nr = nullptr;
  cudaEvent_t ev_ref = nullptr, ev_qkeys = nullptr;
  // X-drop, bands, score pass and gate over the accumulated hits.
  void process_hits(uint64_t pass_id);
  // Hits of the chunks joined since the last process_hits (device, from the
  // context's pool; grows keeping its contents).
  uint64_t* acc = nullptr;
  uint64_t acc_n = 0, acc_cap = 0;
  void acc_reserve(uint64_t n);
  ~Search() {
    if (early_ref) cudaStreamSynchronize(c->side);  // unconsumed side-stream work (a search that stopped early)
    if (acc) cudaFreeAsync(acc, c->stream);
    if (ev_ref) cudaEventDestroy(ev_ref);
    if (ev_qkeys) cudaEventDestroy(ev_qkeys);
  }
  void finish(drg_result* out);
};

void Search::query_seeds(uint64_t* n_runs_out) {
  const int S = (int)shapes.size();
  const uint64_t N = q->total * (uint64_t)S;
  uint32_t* vals = c->q_vals.as<uint32_t>(N);
  uint32_t* vals_s = c->q_vals_s.as<uint32_t>(N);
  uint64_t* rk = c->run_keys.as<uint64_t>(N + 1);
  uint32_t* rc = c->run_counts.as<uint32_t>(N + 1);
  int64_t* h = c->h_stage.as<int64_t>(2);
  uint64_t n_runs = 0;
  // A seed key of at most 32 bits (and no request ids above it) is sorted as
  // a 32-bit key: 8 bytes per entry and pass instead of 12.  The sorted
  // values stay in q_vals_s (the join reads them there); run keys are kept
  // as 64-bit words either way.
  if (!q->request && seed_key_bits <= 32) {
    uint32_t* keys = c->q_keys.as<uint32_t>(N);
    uint32_t* keys_s = c->q_keys_s.as<uint32_t>(N);
    // with the early reference side, the enumeration also sets the query-key
    // bitmap (the same key set as the sorted runs)
    const bool early = early_possible();
    if (early) {
      int lg = 20;
      while (lg < 29 && (1ull << lg) < 24 * N) ++lg;
      const uint64_t words = (1ull << lg) / 32;
      key_filter = c->seed_filter.as<uint32_t>(words);
      key_filter_log2 = lg;
      DRG_CUDA(cudaMemsetAsync(key_filter, 0, words * sizeof(uint32_t), c->stream));
    }
    launch_seed_enum(q->letters, q->offsets, q->owner, 0, q->total, S, keys, vals, c->slot, c->stream,
                     early ? key_filter : nullptr, key_filter_log2);
    if (early) start_early_ref();
    const SortResult<uint32_t> r = dsort(c, keys, keys_s, vals, vals_s, N, 0, seed_key_bits);
    if (r.vals != vals_s) c->q_vals.swap(c->q_vals_s);
    if (N > 0) {
      uint32_t* rk32 = c->run_keys32.as<uint32_t>(N + 1);
      cub_call(c, [&](void* t, size_t& b) {
        return cub::DeviceRunLengthEncode::Encode(t, b, r.keys, rk32, rc, d_count, (int64_t)N, c->stream);
      });
      count_launch();
      k_valid_runs<uint32_t><<<1, 1, 0, c->stream>>>(r.keys, N, rk32, d_count);
      DRG_CUDA(cudaMemcpyAsync(h, d_count, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
      DRG_CUDA(cudaStreamSynchronize(c->stream));
      n_runs = (uint64_t)h[0];
      st.query_seeds = (uint64_t)h[1];
      if (n_runs > 0) {
        count_launch();
        k_widen_keys<<<ceil_div(n_runs, 256), 256, 0, c->stream>>>(rk32, n_runs, rk);
      }
    }
  } else {
    uint64_t* keys = c->q_keys.as<uint64_t>(N);
    uint64_t* keys_s = c->q_keys_s.as<uint64_t>(N);
    launch_seed_enum(q->letters, q->offsets, q->owner, 0, q->total, S, keys, vals, c->slot, c->stream, q->request);
    // request ids sit above the seed key: the sort covers their field up to
    // the batch's largest id ("no seed" keys, all ones, still sort last: a
    // valid key's shape field has a zero bit)
    const int key_bits = q->request ? std::min(64, seed_key_bits + bits_for(q->max_request)) : seed_key_bits;
    const SortResult<uint64_t> r = dsort(c, keys, keys_s, vals, vals_s, N, 0, key_bits);
    if (r.vals != vals_s) c->q_vals.swap(c->q_vals_s);
    // runs of every key (the "no seed" keys, last, form one run of their own),
    // then the valid keys and their runs counted in one kernel: one wait
    if (N > 0) {
      cub_call(c, [&](void* t, size_t& b) {
        return cub::DeviceRunLengthEncode::Encode(t, b, r.keys, rk, rc, d_count, (int64_t)N, c->stream);
      });
      count_launch();
      k_valid_runs<uint64_t><<<1, 1, 0, c->stream>>>(r.keys, N, rk, d_count);
      DRG_CUDA(cudaMemcpyAsync(h, d_count, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
      DRG_CUDA(cudaStreamSynchronize(c->stream));
      n_runs = (uint64_t)h[0];
      st.query_seeds = (uint64_t)h[1];
    }
  }
  uint32_t* qs = c->run_qstart.as<uint32_t>(n_runs + 1);
  if (n_runs > 0)
    cub_call(c, [&](void* t, size_t& b) {
      return cub::DeviceScan::ExclusiveSum(t, b, rc, qs, (int64_t)n_runs, c->stream);
    });
  *n_runs_out = n_runs;
}

// Chunks are joined one by one (the join cap counts reference occurrences
// per chunk, search.rs:127-131), but a subject lives in one chunk, so the
// stages after the join treat every (target, subject) pair on its own: the
// hits of all chunks go through them in one pass (up to a hit budget), which
// saves a pass of fixed launch and sync costs per chunk.
void Search::acc_reserve(uint64_t n) {
  if (n <= acc_cap) return;
  const uint64_t cap = std::max<uint64_t>(n, 2 * acc_cap);
  uint64_t* p = nullptr;
  DRG_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), cap * sizeof(uint64_t), c->pool, c->stream));
  if (acc_n) DRG_CUDA(cudaMemcpyAsync(p, acc, acc_n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, c->stream));
  if (acc) DRG_CUDA(cudaFreeAsync(acc, c->stream));
  acc = p;
  acc_cap = cap;
}

// At least 32 bits per query run up to 2^29 bits (64 MB): then at most 3.1 %
// of the keys that no query holds pass, and the bitmap stays resident in L2
// while the reference seeds probe it.
bool Search::early_possible() const {
  const bool cached = db->cache && db->cache->budget() > 0;
  if (cached || q->request || seed_key_bits > 32 || db->n == 0) return false;
  const auto ch = split_chunks(db->n, index_chunks);
  if (ch.empty()) return false;
  const uint64_t n_pos = (db->h_offsets[ch[0].second] - db->h_offsets[ch[0].first]) * (uint64_t)shapes.size();
  return n_pos < (1ull << 32);
}

void Search::start_early_ref() {
  if (!ev_qkeys) {
    DRG_CUDA(cudaEventCreateWithFlags(&ev_qkeys, cudaEventDisableTiming));
    DRG_CUDA(cudaEventCreateWithFlags(&ev_ref, cudaEventDisableTiming));
  }
  const auto ch = split_chunks(db->n, index_chunks);
  early_c0 = ch[0].first;
  early_c1 = ch[0].second;
  const int S = (int)shapes.size();
  const uint64_t lo = db->h_offsets[early_c0], hi = db->h_offsets[early_c1];
  const uint64_t N = (hi - lo) * (uint64_t)S;
  // every buffer first, on the host (a reallocation would wait for the device)
  unsigned long long* cnt = c->seed_counts.as<unsigned long long>(2);
  uint32_t* vals = c->r_vals.as<uint32_t>(N);
  uint32_t* vs = c->r_vals_s.as<uint32_t>(N);
  uint32_t* k32 = c->r_keys.as<uint32_t>(N);
  uint32_t* ks32 = c->r_keys_s.as<uint32_t>(N);
  uint32_t* err = c->sort_err.as<uint32_t>(1);
  // the query seeds are enumerated and the bitmap set
  DRG_CUDA(cudaEventRecord(ev_qkeys, c->stream));
  DRG_CUDA(cudaStreamWaitEvent(c->side, ev_qkeys, 0));
  // the first chunk's reference seeds the queries can join, sorted on their
  // device-side count with the side stream's sort scratch
  DRG_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), c->side));
  launch_seed_enum_filtered(db->letters, db->offsets, db->owner + lo, lo, hi, S, key_filter, key_filter_log2, k32, vals,
                            cnt, c->slot, c->side);
  count_launch();
  k_add_u64<<<1, 1, 0, c->side>>>(d_counters + 7, cnt + 1);
  const uint64_t* d_nr = reinterpret_cast<const uint64_t*>(cnt);
  const SortResult<uint32_t> r = radix_sort<uint32_t>(k32, ks32, vals, vs, N, d_nr, 0, seed_key_bits, c->sort_tmp_side,
                                                      err, c->side, c->tuning.sort_small_tiles != 0);
  DRG_CUDA(cudaEventRecord(ev_ref, c->side));
  early_keys32_s = r.keys;
  early_vals_s = r.vals;
  early_nr = (int64_t)N;  // capacity; the count is d_nr
  early_d_nr = d_nr;
  early_ref = true;
}

void Search::build_key_filter(uint64_t n_runs) {
  int lg = 20;
  while (lg < 29 && (1ull << lg) < 32 * n_runs) ++lg;
  const uint64_t words = (1ull << lg) / 32;
  key_filter = c->seed_filter.as<uint32_t>(words);
  DRG_CUDA(cudaMemsetAsync(key_filter, 0, words * sizeof(uint32_t), c->stream));
  launch_key_filter(c->run_keys.as<uint64_t>(0), n_runs, (1ull << seed_key_bits) - 1, key_filter, lg, c->stream);
  key_filter_log2 = lg;
}

void Search::join_chunk(uint64_t c0, uint64_t c1, uint64_t n_runs) {
  Timer tm(c, &times);
  const int S = (int)shapes.size();
  const uint64_t lo = db->h_offsets[c0], hi = db->h_offsets[c1];
  const uint64_t N = (hi - lo) * (uint64_t)S;
  // ---- reference seeds (or the database's cached index of them) + join
  tm.start();
  IndexCache* cache = db->cache && db->cache->budget() > 0 ? db->cache.get() : nullptr;
  const std::string ikey = cache ? index_key(c0, c1) : std::string();
  std::shared_ptr<SeedIndex> held = cache ? cache->find(ikey) : nullptr;  // kept until the join has read it
  // A seed key of at most 32 bits is sorted as a 32-bit key: 8 bytes per
  // entry and pass instead of 12.
  const bool key32 = seed_key_bits <= 32;
  const uint64_t* keys_s = nullptr;
  const uint32_t* keys32_s = nullptr;
  const uint32_t* vals_s;
  int64_t nr;             // reference seeds the join reads (a bound when d_nr is set)
  const uint64_t* d_nr = nullptr;  // their count on the device, when the host does not know it
  uint64_t n_valid = 0;   // valid reference seeds of the chunk (counted on the device when d_nr is set)
  if (held) {
    keys_s = held->keys;
    keys32_s = held->keys32;
    vals_s = held->vals;
    nr = (int64_t)held->n;
    n_valid = held->n;
    st.index_hits += 1;
  } else if (!cache && early_ref && c0 == early_c0 && c1 == early_c1) {
    // sorted on the side stream while the query seeds sorted
    DRG_CUDA(cudaStreamWaitEvent(c->stream, ev_ref, 0));
    early_ref = false;
    keys32_s = early_keys32_s;
    vals_s = early_vals_s;
    nr = early_nr;
    d_nr = early_d_nr;
  } else if (!cache) {
    // Nothing is kept for later searches, so only the seeds whose key the
    // query holds are sorted: the join pairs equal keys only (seed.rs:110-140),
    // so the rest cannot yield a hit or change a run's count.
    if (!key_filter) build_key_filter(n_runs);
    unsigned long long* cnt = c->seed_counts.as<unsigned long long>(2);
    DRG_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), c->stream));
    uint32_t* vals = c->r_vals.as<uint32_t>(N);
    uint32_t* vs = c->r_vals_s.as<uint32_t>(N);
    uint32_t *k32 = nullptr, *ks32 = nullptr;
    uint64_t *k64 = nullptr, *ks64 = nullptr;
    if (key32) {
      k32 = c->r_keys.as<uint32_t>(N);
      ks32 = c->r_keys_s.as<uint32_t>(N);
      launch_seed_enum_filtered(db->letters, db->offsets, db->owner + lo, lo, hi, S, key_filter, key_filter_log2, k32,
                                vals, cnt, c->slot, c->stream);
    } else {
      k64 = c->r_keys.as<uint64_t>(N);
      ks64 = c->r_keys_s.as<uint64_t>(N);
      launch_seed_enum_filtered(db->letters, db->offsets, db->owner + lo, lo, hi, S, key_filter, key_filter_log2, k64,
                                vals, cnt, c->slot, c->stream);
    }
    // the kept count stays on the device: the sort, the bucket starts and the
    // join read it there (no host wait); the valid count joins the counters.
    // A chunk with more seed positions than one sort takes (2^32 - 1) reads
    // the kept count first (the kept seeds are the ones its queries can join).
    count_launch();
    k_add_u64<<<1, 1, 0, c->stream>>>(d_counters + 7, cnt + 1);
    uint64_t n_sort = N;
    if (N < (1ull << 32)) {
      d_nr = reinterpret_cast<const uint64_t*>(cnt);
      nr = (int64_t)N;  // capacity
    } else {
      nr = (int64_t)fetch(c, cnt);
      n_sort = (uint64_t)nr;
    }
    if (key32) {
      const SortResult<uint32_t> r = dsort(c, k32, ks32, vals, vs, n_sort, 0, seed_key_bits, d_nr);
      ks32 = r.keys;
      vs = r.vals;
    } else {
      const SortResult<uint64_t> r = dsort(c, k64, ks64, vals, vs, n_sort, 0, seed_key_bits, d_nr);
      ks64 = r.keys;
      vs = r.vals;
    }
    keys_s = ks64;
    keys32_s = ks32;
    vals_s = vs;
  } else {
    uint32_t* vals = c->r_vals.as<uint32_t>(N);
    uint32_t* vs = c->r_vals_s.as<uint32_t>(N);
    if (key32) {
      uint32_t* keys = c->r_keys.as<uint32_t>(N);
      uint32_t* ks = c->r_keys_s.as<uint32_t>(N);
      launch_seed_enum(db->letters, db->offsets, db->owner + lo, lo, hi, S, keys, vals, c->slot, c->stream);
      const SortResult<uint32_t> r = dsort(c, keys, ks, vals, vs, N, 0, seed_key_bits);
      ks = r.keys;
      vs = r.vals;
      nr = count_valid(c, ks, N, d_count);
      keys32_s = ks;
    } else {
      uint64_t* keys = c->r_keys.as<uint64_t>(N);
      uint64_t* ks = c->r_keys_s.as<uint64_t>(N);
      launch_seed_enum(db->letters, db->offsets, db->owner + lo, lo, hi, S, keys, vals, c->slot, c->stream);
      const SortResult<uint64_t> r = dsort(c, keys, ks, vals, vs, N, 0, seed_key_bits);
      ks = r.keys;
      vs = r.vals;
      nr = count_valid(c, ks, N, d_count);
      keys_s = ks;
    }
    vals_s = vs;
    n_valid = (uint64_t)nr;
    held = cache->insert(ikey, keys_s, keys32_s, vs, (uint64_t)nr, c->stream);
  }
  st.ref_seeds += n_valid;
  uint32_t* rlo = c->run_rlo.as<uint32_t>(n_runs + 1);
  uint32_t* rcnt = c->run_rcount.as<uint32_t>(n_runs + 1);
  uint64_t* rhits = c->run_hits.as<uint64_t>(n_runs + 1);
  uint64_t* roff = c->run_hit_off.as<uint64_t>(n_runs + 1);
  // bucket starts over the top 16 bits of the sorted reference keys: each
  // query run then searches ~nr / 65536 keys instead of nr
  const int bucket_bits = std::min(16, seed_key_bits);
  const int shift = seed_key_bits - bucket_bits;
  const uint32_t nb = 1u << bucket_bits;
  uint32_t* first = c->ref_first.as<uint32_t>(nb + 1);
  if (keys32_s) {
    launch_bucket_first(keys32_s, (uint64_t)nr, shift, nb, first, c->stream, d_nr);
    launch_join_count(c->run_keys.as<uint64_t>(0), c->run_counts.as<uint32_t>(0), n_runs, keys32_s, (uint64_t)nr,
                      4096, rlo, rcnt, rhits, (1ull << seed_key_bits) - 1, c->stream, first, shift, nullptr, d_nr);
  } else {
    launch_bucket_first(keys_s, (uint64_t)nr, shift, nb, first, c->stream, d_nr);
    launch_join_count(c->run_keys.as<uint64_t>(0), c->run_counts.as<uint32_t>(0), n_runs, keys_s, (uint64_t)nr, 4096,
                      rlo, rcnt, rhits, (1ull << seed_key_bits) - 1, c->stream, first, shift, nullptr, d_nr);
  }
  // hits of the runs' entries in [qstart, +count) (all, or one block's)
  auto scan_hits = [&]() {
    count_launch();
    k_set_u64<<<1, 1, 0, c->stream>>>(rhits + n_runs, 0);
    cub_call(c, [&](void* t, size_t& b) {
      return cub::DeviceScan::ExclusiveSum(t, b, rhits, roff, (int64_t)n_runs + 1, c->stream);
    });
    return fetch(c, roff + n_runs);
  };
  auto expand = [&](uint64_t n_hits, const uint32_t* qstart) {
    st.hits += n_hits;
    acc_reserve(acc_n + n_hits);
    if (n_hits > 0) {
      JoinExpandArgs ja{};
      ja.run_hit_off = roff;
      ja.coarse_shift = 7;  // one entry per 128 hits
      uint32_t* coarse = c->hit_coarse.as<uint32_t>(((n_hits - 1) >> ja.coarse_shift) + 2);
      launch_hit_coarse(roff, n_runs, ja.coarse_shift, n_hits, coarse, c->stream);
      ja.coarse = coarse;
      ja.run_qstart = qstart;
      ja.run_rlo = rlo;
      ja.run_rcount = rcnt;
      ja.n_runs = n_runs;
      ja.q_vals = c->q_vals_s.as<uint32_t>(0);
      ja.r_vals = vals_s;
      ja.n_hits = n_hits;
      ja.q_owner = q->owner;
      ja.q_offsets = q->offsets;
      ja.r_owner = db->owner;
      ja.r_offsets = db->offsets;
      ja.layout = layout();
      ja.hit_keys = acc + acc_n;
      launch_join_expand(ja, c->stream);
    }
    acc_n += n_hits;
  };
  const uint64_t n_hits = scan_hits();
  if ((n_hits <= hit_budget || q->n == 1) && q->n <= t_window) {
    // the stages after the join run on hits of several chunks at once, up to
    // the budget (a subject lives in one chunk: pairs never span passes)
    if (acc_n > 0 && acc_n + n_hits > hit_budget) {
      tm.stop(&st.ms_join);
      process_hits(pass++);
      tm.start();
    }
    expand(n_hits, c->run_qstart.as<uint32_t>(0));
    ++query_blocks;
    tm.stop(&st.ms_join);
    return;
  }
  // ---- query blocks: consecutive targets whose hits stay under the budget
  // and that fit one target window of the hit key (a target is never split:
  // its pairs are then all in one pass)
  unsigned long long* thits = c->target_hits.as<unsigned long long>(q->n);
  DRG_CUDA(cudaMemsetAsync(thits, 0, q->n * sizeof(unsigned long long), c->stream));
  launch_target_hits(c->run_counts.as<uint32_t>(0), c->run_qstart.as<uint32_t>(0), rcnt, rhits, n_runs,
                     c->q_vals_s.as<uint32_t>(0), q->owner, thits, c->stream);
  std::vector<unsigned long long> th;
  fetch_n(c, th, thits, q->n);
  std::vector<std::pair<uint64_t, uint64_t>> blocks;
  for (uint64_t t0 = 0; t0 < q->n;) {
    uint64_t t1 = t0, sum = 0;
    while (t1 < q->n && t1 - t0 < t_window && (t1 == t0 || sum + th[t1] <= hit_budget)) sum += th[t1++];
    blocks.push_back({t0, t1});
    t0 = t1;
  }
  if (acc_n > 0) {
    tm.stop(&st.ms_join);
    process_hits(pass++);
    tm.start();
  }
  uint32_t* qlo = c->run_qlo.as<uint32_t>(n_runs + 1);
  uint32_t* qcnt = c->run_qcount.as<uint32_t>(n_runs + 1);
  for (auto [t0, t1] : blocks) {
    t_base = t0;  // the hit keys of this block (expand, then process_hits)
    JoinBlock jb{c->q_vals_s.as<uint32_t>(0), c->run_qstart.as<uint32_t>(0), q->h_offsets[t0], q->h_offsets[t1], qlo,
                 qcnt};
    const uint64_t key_mask = (1ull << seed_key_bits) - 1;
    if (keys32_s)
      launch_join_count(c->run_keys.as<uint64_t>(0), c->run_counts.as<uint32_t>(0), n_runs, keys32_s, (uint64_t)nr,
                        4096, rlo, rcnt, rhits, key_mask, c->stream, first, shift, &jb, d_nr);
    else
      launch_join_count(c->run_keys.as<uint64_t>(0), c->run_counts.as<uint32_t>(0), n_runs, keys_s, (uint64_t)nr,
                        4096, rlo, rcnt, rhits, key_mask, c->stream, first, shift, &jb, d_nr);
    expand(scan_hits(), qlo);
    ++query_blocks;
    tm.stop(&st.ms_join);
    process_hits(pass++);
    tm.start();
  }
  t_base = 0;
  tm.stop(&st.ms_join);
}

void Search::process_hits(uint64_t pass_id) {
  Timer tm(c, &times);
  const uint64_t n_hits = acc_n;
  acc_n = 0;
  if (n_hits == 0) return;
  const HitKeyLayout L = layout();
  const uint64_t* hk = acc;
  // The stages up to the score pass run on counts that stay on the device
  // (unique hits, diagonal runs, kept segments, pairs, bands), each bounded
  // by n_hits: every buffer is sized for n_hits, each kernel reads its count
  // from dc, and one wait at the end reads them all.
  //   dc[0] unique hits  [1] diagonal runs  [2] kept segments  [3] pairs
  //   [4] bands  [5] pair starts
  int64_t* dc = c->pass_counts.as<int64_t>(8);
  DRG_CUDA(cudaMemsetAsync(dc, 0, 8 * sizeof(int64_t), c->stream));
  // ---- sort + unique hits
  tm.start();
  uint64_t* hs = c->hits_s.as<uint64_t>(n_hits);
  uint64_t* hu = c->hits_u.as<uint64_t>(n_hits);
  hs = dsort<uint64_t>(c, const_cast<uint64_t*>(hk), hs, nullptr, nullptr, n_hits, 0, L.total()).keys;
  cub_call(c, [&](void* t, size_t& b) {
    return cub::DeviceSelect::Unique(t, b, hs, hu, dc + 0, (int64_t)n_hits, c->stream);
  });
  tm.stop(&st.ms_sort);
  // ---- ungapped
  tm.start();
  uint8_t* flags = c->flags.as<uint8_t>(n_hits + 1);
  uint32_t* idx = c->idx.as<uint32_t>(n_hits + 1);
  launch_run_heads(hu, n_hits, L.pb, flags, c->stream, dc + 0);
  select_indices_dev(c, flags, n_hits, idx, dc + 1);
  SegmentOut* segs = c->segs.as<SegmentOut>(n_hits);
  uint8_t* keep = c->keep.as<uint8_t>(n_hits);
  DRG_CUDA(cudaMemsetAsync(keep, 0, n_hits, c->stream));  // past the unique hits: not kept
  XdropArgs xa{};
  xa.hit_keys = hu;
  xa.n_hits = n_hits;
  xa.run_head_idx = idx;
  xa.n_runs = n_hits;
  xa.d_n_hits = dc + 0;
  xa.d_n_runs = dc + 1;
  xa.layout = L;
  xa.q_letters = q->letters;
  xa.q_offsets = q->offsets;
  xa.s_letters = db->letters;
  xa.s_offsets = db->offsets;
  xa.xdrop = sc.raw_score(12.3);
  xa.cutoff = 19;
  xa.seg = segs;
  xa.keep = keep;
  xa.xdrop_count = d_counters + 0;
  xa.slot = c->slot;
  launch_xdrop_runs(xa, c->stream);
  uint64_t* sk = c->seg_keys.as<uint64_t>(n_hits);
  SegmentOut* sc_ = c->segs_c.as<SegmentOut>(n_hits);
  cub_call(c, [&](void* t, size_t& b) {
    return cub::DeviceSelect::Flagged(t, b, hu, keep, sk, dc + 2, (int64_t)n_hits, c->stream);
  });
  cub_call(c, [&](void* t, size_t& b) {
    return cub::DeviceSelect::Flagged(t, b, segs, keep, sc_, dc + 2, (int64_t)n_hits, c->stream);
  });
  tm.stop(&st.ms_ungapped);
  // ---- bands
  tm.start();
  launch_run_heads(sk, n_hits, L.pb + L.db, flags, c->stream, dc + 2);
  select_indices_dev(c, flags, n_hits, idx, dc + 3);
  count_launch();
  k_set_at<<<1, 1, 0, c->stream>>>(idx, dc + 3, dc + 2);  // idx[pairs] = segments
  Band* bands = c->bands.as<Band>(n_hits);
  uint8_t* bvalid = c->band_valid.as<uint8_t>(n_hits);
  DRG_CUDA(cudaMemsetAsync(bvalid, 0, n_hits, c->stream));
  BandArgs ba{};
  ba.seg_keys = sk;
  ba.segs = sc_;
  ba.n_segs = n_hits;
  ba.pair_head_idx = idx;
  ba.n_pairs = n_hits;
  ba.d_n_pairs = dc + 3;
  ba.layout = L;
  ba.q_offsets = q->offsets;
  ba.bands = bands;
  ba.valid = bvalid;
  launch_build_bands(ba, c->stream);
  Band* bc = c->bands_c.as<Band>(n_hits);
  cub_call(c, [&](void* t, size_t& b) {
    return cub::DeviceSelect::Flagged(t, b, bands, bvalid, bc, dc + 4, (int64_t)n_hits, c->stream);
  });
  uint32_t* pfirst = c->pair_first.as<uint32_t>(n_hits + 1);
  count_launch();
  k_rank0_flags_dev<<<ceil_div(n_hits, 256), 256, 0, c->stream>>>(bc, n_hits, dc + 4, flags);
  select_indices_dev(c, flags, n_hits, pfirst, dc + 5);
  count_launch();
  k_set_at<<<1, 1, 0, c->stream>>>(pfirst, dc + 3, dc + 4);  // pfirst[pairs] = bands
  // the one wait of these stages: their counts
  int64_t* hc = c->h_stage.as<int64_t>(8);
  DRG_CUDA(cudaMemcpyAsync(hc, dc, 8 * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  DRG_CUDA(cudaStreamSynchronize(c->stream));
  const uint64_t n_u = (uint64_t)hc[0], n_segs = (uint64_t)hc[2], n_pairs = (uint64_t)hc[3],
                 n_bands = (uint64_t)hc[4];
  st.unique_hits += n_u;
  st.segments += n_segs;
  st.bands += n_bands;
  tm.stop(&st.ms_bands);
  if (n_segs == 0 || n_bands == 0) return;
  // ---- banded SW scores
  tm.start();
  int32_t* scores = c->scores.as<int32_t>(n_bands);
  DevSeqs qs{q->letters, q->offsets, &q->h_offsets, q->score_letters};
  DevSeqs ss{db->letters, db->offsets, &db->h_offsets, db->score_letters};
  int32_t* best_row = c->best_row.as<int32_t>(n_bands);
  run_bands(c, bc, n_bands, qs, ss, sc, false, scores, best_row, nullptr, nullptr, nullptr, nullptr, st, d_count,
            d_counters + 3, &times);
  tm.stop(&st.ms_sw);
  flags = c->flags.as<uint8_t>(n_bands + 1);  // scratch buffers may have been regrown
  // ---- E-value gate and band walk
  tm.start();
  uint8_t* state = c->state.as<uint8_t>(n_bands);
  SelectArgs ga{};
  ga.bands = bc;
  ga.score = scores;
  ga.n_bands = n_bands;
  ga.pair_first = pfirst;
  ga.n_pairs = n_pairs;
  ga.q_offsets = q->offsets;
  ga.s_offsets = db->offsets;
  ga.db_letters = db->total;
  const Alp& A = sc.alp;
  ga.alp = AlpDev{A.lambda, A.k, A.ln_k, A.a, A.b, A.alpha, A.beta, A.sigma, A.tau, A.v_thr, A.c_thr};
  ga.evalue = evalue;
  ga.max_hsps = (uint32_t)std::min<uint64_t>(max_hsps, 0xFFFFFFFFu);
  ga.state = state;
  ga.verdict = c->verdict.as<uint8_t>(n_bands);
  ga.cells_ref = d_counters + 1;
  ga.n_computed = d_counters + 2;
  launch_select(ga, c->stream);
  count_launch();
  k_state_flags<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(state, n_bands, flags);
  // the kept and undecided bands, gathered on their device-side count: one
  // wait for the count, one for the records (pinned staging)
  uint32_t* sel = c->sel_idx.as<uint32_t>(n_bands + 1);
  int64_t* dsel = c->pass_counts.as<int64_t>(8) + 6;
  select_indices_dev(c, flags, n_bands, sel, dsel);
  Band* gb = c->sel_bands.as<Band>(n_bands);
  int32_t* gs = reinterpret_cast<int32_t*>(c->exact_out.as<uint8_t>(n_bands * 5 + 16));
  uint8_t* gst = reinterpret_cast<uint8_t*>(gs + n_bands);
  count_launch();
  k_gather_bands_dev<<<ceil_div(n_bands, 256), 256, 0, c->stream>>>(sel, n_bands, dsel, bc, scores, best_row, state,
                                                                      gb, gs, gst);
  const uint64_t n_sel = (uint64_t)fetch(c, dsel);
  if (n_sel > 0) {
    const size_t rec = sizeof(Band) + sizeof(int32_t) + 1;
    uint8_t* h = c->h_stage.as<uint8_t>(n_sel * rec + 16);
    Band* hb = reinterpret_cast<Band*>(h);
    int32_t* hs_ = reinterpret_cast<int32_t*>(h + n_sel * sizeof(Band));
    uint8_t* hst = reinterpret_cast<uint8_t*>(hs_ + n_sel);
    DRG_CUDA(cudaMemcpyAsync(hb, gb, n_sel * sizeof(Band), cudaMemcpyDeviceToHost, c->stream));
    DRG_CUDA(cudaMemcpyAsync(hs_, gs, n_sel * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DRG_CUDA(cudaMemcpyAsync(hst, gst, n_sel, cudaMemcpyDeviceToHost, c->stream));
    DRG_CUDA(cudaStreamSynchronize(c->stream));
    for (uint64_t k = 0; k < n_sel; ++k) {
      Candidate cd;
      cd.band = hb[k];
      cd.score = hs_[k];
      cd.state = hst[k];
      cd.pair_key = (pass_id << 32) | hb[k].pair;
      cd.evalue = 0;
      cd.bits = 0;
      cands.push_back(cd);
    }
  }
  tm.stop(&st.ms_select);
}

int cmp_cand(const Candidate& a, const Candidate& b) {  // cmp_hsp, search.rs:273-282
  if (a.score != b.score) return b.score < a.score ? -1 : 1;
  if (a.evalue < b.evalue) return -1;
  if (a.evalue > b.evalue) return 1;
  if (a.band.subject != b.band.subject) return a.band.subject < b.band.subject ? -1 : 1;
  return 0;
}

void Search::finish(drg_result* out) {
  auto t0 = std::chrono::steady_clock::now();
  // The exact host E-values (glibc libm, like the reference) of every
  // candidate, on the context's host threads: a pure function of (score,
  // qlen, slen), used below in the reference's order.
  std::vector<double> ev(cands.size(), 0.0);
  {
    if (!c->host_pool) {
      const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
      c->host_pool.reset(new host::Pool(std::min(hw - 1, 15u)));
    }
    c->host_pool->parallel_for(cands.size(), 256, host_threads, [&](uint64_t lo, uint64_t hi) {
      for (uint64_t k = lo; k < hi; ++k) {
        const Candidate& cd = cands[k];
        if (cd.score <= 0) continue;
        const uint64_t qlen = q->h_offsets[cd.band.target + 1] - q->h_offsets[cd.band.target];
        const uint64_t slen = db->h_offsets[cd.band.subject + 1] - db->h_offsets[cd.band.subject];
        ev[k] = sc.evalue(cd.score, qlen, slen, db->total);
      }
    });
  }
  // exact statistics and the walk of undecided pairs
  std::vector<Candidate> kept;
  kept.reserve(cands.size());
  for (size_t i = 0; i < cands.size();) {
    size_t j = i;
    while (j < cands.size() && cands[j].pair_key == cands[i].pair_key) ++j;
    uint64_t nkept = 0;
    for (size_t k = i; k < j; ++k) {
      Candidate cd = cands[k];
      if (cd.state == 2) {
        cd.evalue = ev[k];
        cd.bits = sc.bit_score(cd.score);
        kept.push_back(cd);
        ++nkept;
      } else {  // undecided: continue the reference's walk exactly
        if (nkept >= max_hsps) continue;
        if (cd.score <= 0) continue;
        const double e = ev[k];
        if (e <= evalue) {
          cd.evalue = e;
          cd.bits = sc.bit_score(cd.score);
          cd.state = 2;
          kept.push_back(cd);
          ++nkept;
        }
      }
    }
    i = j;
  }
  // per target: pairs in subject order, HSPs of a pair by cmp_hsp, pairs by
  // their best HSP, then --max-target-seqs and --max-hsps (search.rs:256-270).
  // One index array, stably ordered by (target, subject); each pair's HSPs
  // sorted in place by cmp_hsp; each target's pairs then ordered by their
  // best HSP (stable).  No per-target containers: the culling is linear
  // after the sorts.
  std::vector<uint32_t> idx(kept.size());
  for (size_t k = 0; k < kept.size(); ++k) idx[k] = (uint32_t)k;
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
    const Band &x = kept[a].band, &y = kept[b].band;
    return x.target != y.target ? x.target < y.target : x.subject < y.subject;
  });
  std::vector<std::pair<uint32_t, uint32_t>> pairs;  // [begin, end) ranges of idx, one per (target, subject)
  for (size_t i = 0; i < idx.size();) {
    size_t j = i;
    const Band& bi = kept[idx[i]].band;
    while (j < idx.size() && kept[idx[j]].band.target == bi.target && kept[idx[j]].band.subject == bi.subject) ++j;
    std::stable_sort(idx.begin() + i, idx.begin() + j,
                     [&](uint32_t a, uint32_t b) { return cmp_cand(kept[a], kept[b]) < 0; });
    pairs.push_back({(uint32_t)i, (uint32_t)j});
    i = j;
  }
  std::vector<size_t> order;
  std::vector<uint64_t> final_off(q->n + 1, 0);
  for (size_t pp = 0, t = 0; t < q->n; ++t) {
    size_t p1 = pp;
    while (p1 < pairs.size() && kept[idx[pairs[p1].first]].band.target == t) ++p1;
    std::stable_sort(pairs.begin() + pp, pairs.begin() + p1,
                     [&](const std::pair<uint32_t, uint32_t>& a, const std::pair<uint32_t, uint32_t>& b) {
                       return cmp_cand(kept[idx[a.first]], kept[idx[b.first]]) < 0;
                     });
    const size_t np = std::min<size_t>(p1 - pp, max_targets);
    for (size_t g = pp; g < pp + np; ++g) {
      const size_t len = std::min<size_t>(pairs[g].second - pairs[g].first, max_hsps);
      for (size_t e = 0; e < len; ++e) order.push_back(idx[pairs[g].first + e]);
    }
    final_off[t + 1] = order.size();
    pp = p1;
  }
  // traceback for the survivors
  const uint64_t nj = order.size();
  std::vector<Band> sb(nj);
  std::vector<uint64_t> ops_off(nj + 1, 0);
  for (uint64_t k = 0; k < nj; ++k) {
    sb[k] = kept[order[k]].band;
    const uint64_t m = db->h_offsets[sb[k].subject + 1] - db->h_offsets[sb[k].subject];
    ops_off[k + 1] = ops_off[k] + sb[k].n + m;
  }
  st.ms_host += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  std::vector<ExactOut> eo;
  std::vector<uint32_t> ops_all;
  if (nj > 0) {
    Timer tm(c, &times);
    tm.start();
    Band* db_ = c->sel_bands.as<Band>(nj);
    uint64_t* doff = c->ops_off.as<uint64_t>(nj + 1);
    ExactOut* dout = c->trace_out.as<ExactOut>(nj);
    uint32_t* dops = c->exact_ops.as<uint32_t>(ops_off[nj] + 1);
    DRG_CUDA(cudaMemcpyAsync(db_, sb.data(), nj * sizeof(Band), cudaMemcpyHostToDevice, c->stream));
    DRG_CUDA(cudaMemcpyAsync(doff, ops_off.data(), (nj + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    DevSeqs qs{q->letters, q->offsets, &q->h_offsets, q->score_letters};
    DevSeqs ss{db->letters, db->offsets, &db->h_offsets, db->score_letters};
    run_bands(c, db_, nj, qs, ss, sc, true, nullptr, nullptr, dout, dops, doff, &ops_off, st, d_count,
              nullptr, &times);
    // only the ops the alignments use come back (each band has n + m slots)
    uint64_t* cnt = c->ops_cnt.as<uint64_t>(nj + 1);
    uint64_t* coff = c->ops_coff.as<uint64_t>(nj + 1);
    count_launch();
    k_ops_count<<<ceil_div(nj + 1, 256), 256, 0, c->stream>>>(dout, nj, cnt);
    cub_call(c, [&](void* t, size_t& b) {
      return cub::DeviceScan::ExclusiveSum(t, b, cnt, coff, (int64_t)nj + 1, c->stream);
    });
    // compacted into a buffer of the bands' slot total (an upper bound of the
    // ops used); the records and the used count come back in one wait
    uint32_t* cops = c->ops_compact.as<uint32_t>(ops_off[nj] + 1);
    count_launch();
    k_compact_ops<<<ceil_div(nj, 128), 128, 0, c->stream>>>(dops, doff, dout, coff, nj, cops);
    uint8_t* hst = c->h_stage.as<uint8_t>(nj * sizeof(ExactOut) + 16);
    DRG_CUDA(cudaMemcpyAsync(hst, dout, nj * sizeof(ExactOut), cudaMemcpyDeviceToHost, c->stream));
    DRG_CUDA(cudaMemcpyAsync(hst + nj * sizeof(ExactOut), coff + nj, sizeof(uint64_t), cudaMemcpyDeviceToHost,
                             c->stream));
    DRG_CUDA(cudaStreamSynchronize(c->stream));
    eo.assign(reinterpret_cast<const ExactOut*>(hst), reinterpret_cast<const ExactOut*>(hst) + nj);
    uint64_t n_used = 0;
    std::memcpy(&n_used, hst + nj * sizeof(ExactOut), sizeof(uint64_t));
    fetch_n(c, ops_all, cops, n_used);
    tm.stop(&st.ms_trace);
  }
  auto t1 = std::chrono::steady_clock::now();
  // assemble per-target lists
  out->n_targets = q->n;
  out->target_offsets = (uint64_t*)std::malloc(sizeof(uint64_t) * (q->n + 1));
  out->hsps = (drg_hsp*)std::malloc(sizeof(drg_hsp) * (nj + 1));
  uint64_t total_ops = 0;
  for (uint64_t k = 0; k < nj; ++k) total_ops += eo[k].n_ops;
  out->ops = (uint32_t*)std::malloc(sizeof(uint32_t) * (total_ops + 1));
  if (!out->target_offsets || !out->hsps || !out->ops) throw Error(DRG_ERR_OOM, "host allocation failed");
  uint64_t h = 0, ko = 0, k = 0;
  out->target_offsets[0] = 0;
  for (uint64_t t = 0; t < q->n; ++t) {
    for (uint64_t kk = final_off[t]; kk < final_off[t + 1]; ++kk, ++k) {
      const Candidate& cd = kept[order[k]];
      const ExactOut& r = eo[k];
      if (r.score != cd.score)
        throw Error(DRG_ERR_CUDA, "internal: traceback score " + std::to_string(r.score) + " != band score " +
                                      std::to_string(cd.score));
      drg_hsp& o = out->hsps[h++];
      o.query = q->query[t];
      o.subject = cd.band.subject;
      o.frame = q->frame[t];
      o.score = r.score;
      o.q_begin = cd.band.q0 + r.q_begin;
      o.q_end = cd.band.q0 + r.q_end;
      o.s_begin = r.s_begin;
      o.s_end = r.s_end;
      o.bits = cd.bits;
      o.evalue = cd.evalue;
      o.identities = r.identities;
      o.positives = r.positives;
      o.mismatches = r.mismatches;
      o.gap_openings = r.gap_openings;
      o.gaps = r.gaps;
      o.length = r.length;
      o.ops_offset = ko;
      o.n_ops = r.n_ops;
      o.pad = 0;
      std::memcpy(out->ops + ko, ops_all.data() + ko, r.n_ops * sizeof(uint32_t));  // compacted in this order
      ko += r.n_ops;
    }
    out->target_offsets[t + 1] = h;
  }
  out->n_hsps = h;
  out->n_ops = ko;
  st.traced_bands = nj;
  st.hsps = h;
  st.ms_host += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
}

void Search::run(drg_result* out) {
  const uint64_t launches0 = kernel_launch_count();
  Timer total(c, &times);
  total.start();
  std::memset(out, 0, sizeof(*out));
  d_count = c->counters.as<int64_t>(12);
  d_counters = reinterpret_cast<unsigned long long*>(d_count + 2);
  DRG_CUDA(cudaMemsetAsync(d_count, 0, 12 * sizeof(int64_t), c->stream));
  DRG_CUDA(cudaMemsetAsync(c->sort_err.as<uint32_t>(1), 0, sizeof(uint32_t), c->stream));
  if (q->n == 0 || db->n == 0) {
    out->n_targets = q->n;
    out->target_offsets = (uint64_t*)std::calloc(q->n + 1, sizeof(uint64_t));
    out->hsps = (drg_hsp*)std::malloc(sizeof(drg_hsp));
    out->ops = (uint32_t*)std::malloc(sizeof(uint32_t));
    total.stop(&st.ms_total);
    DRG_CUDA(cudaStreamSynchronize(c->stream));
    times.resolve();
    out->stats = st;
    return;
  }
  set_target_window();
  Timer tm(c, &times);
  tm.start();
  uint64_t n_runs = 0;
  query_seeds(&n_runs);
  tm.stop(&st.ms_seed);
  if (n_runs > 0) {
    for (auto [c0, c1] : split_chunks(db->n, index_chunks)) join_chunk(c0, c1, n_runs);
    process_hits(pass++);
  }
  if (early_ref) {  // no join read it: its buffers must not outlive this search's use of them
    DRG_CUDA(cudaStreamWaitEvent(c->stream, ev_ref, 0));
    early_ref = false;
  }
  finish(out);
  total.stop(&st.ms_total);
  unsigned long long cnt[8];
  uint32_t sort_err = 0;
  DRG_CUDA(cudaMemcpyAsync(cnt, d_counters, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
  DRG_CUDA(cudaMemcpyAsync(&sort_err, c->sort_err.as<uint32_t>(1), sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  DRG_CUDA(cudaStreamSynchronize(c->stream));
  if (sort_err) throw Error(DRG_ERR_TIMEOUT, "radix sort: a tile's bounded wait for an earlier tile gave up");
  times.resolve();
  st.xdrops = cnt[0];
  st.dp_cells_ref = cnt[1];
  st.bands_computed = cnt[2];
  st.dp_cells_gpu = cnt[3];
  st.dp_cells_lane = cnt[4];
  st.dp_cells_issued = cnt[5];
  st.sw_transposed_bands = cnt[6];
  st.ref_seeds += cnt[7];  // valid reference seeds counted on the device
  st.seed_shapes = shapes.size();
  st.query_blocks = query_blocks;
  st.hit_passes = pass;
  st.kernel_launches = kernel_launch_count() - launches0;
  out->stats = st;
}

}  // namespace

void search(drg_ctx* ctx, const drg_db* db, const drg_batch* b, const drg_search_config* cfg, drg_result* out) {
  Search s;
  s.c = ctx;
  s.db = db;
  s.q = b;
  s.configure(cfg);
  s.run(out);
  ctx->last = out->stats;
}

// Resident inputs come from the context's stream-ordered pool, which keeps
// freed memory for the next call instead of returning it to the driver.
template <typename T>
static void pool_alloc(drg_ctx* ctx, T** p, size_t bytes) {
  DRG_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, ctx->pool, ctx->stream));
}
static void pool_free(drg_ctx* ctx, void* p) {
  if (p) cudaFreeAsync(p, ctx->stream);
}

bool letters_above_24(drg_ctx* c, const uint8_t* d_letters, uint64_t n) {
  unsigned int* bad = c->letter_check.as<unsigned int>(1);
  launch_check_letters(d_letters, n, bad, c->stream);
  return fetch(c, bad) != 0;
}

// Letter codes above 24 score as 24 (matrix.rs:164-168) while identities
// compare the codes themselves (hsp.rs:46-56): the DP kernels then read a
// clamped copy, everything else the letters as given.
template <typename Obj>
static void clamp_for_dp(drg_ctx* ctx, Obj* o) {
  if (!letters_above_24(ctx, o->letters, o->total)) return;
  pool_alloc(ctx, &o->score_letters, o->total + 64);
  DRG_CUDA(cudaMemsetAsync(o->score_letters + o->total, 25, 64, ctx->stream));
  launch_clamp_letters(o->letters, o->total, o->score_letters, ctx->stream);
  DRG_CUDA(cudaStreamSynchronize(ctx->stream));
}

drg_db* make_db(drg_ctx* ctx, const uint8_t* letters, const uint64_t* offsets, uint64_t n) {
  drg_db* d = new drg_db();
  d->ctx = ctx;
  d->n = n;
  d->h_offsets.assign(offsets, offsets + n + 1);
  d->total = offsets[n];
  for (uint64_t i = 0; i < n; ++i) {
    if (offsets[i + 1] < offsets[i]) {
      delete d;
      throw Error(DRG_ERR_INVALID, "database offsets must be non-decreasing");
    }
    d->max_len = std::max<uint32_t>(d->max_len, (uint32_t)(offsets[i + 1] - offsets[i]));
  }
  d->cache.reset(new IndexCache(ctx->device));
  try {
    pool_alloc(ctx, &d->letters, d->total + 64);
    pool_alloc(ctx, &d->offsets, (n + 1) * sizeof(uint64_t));
    pool_alloc(ctx, &d->owner, (d->total + 1) * sizeof(uint32_t));
    DRG_CUDA(cudaMemsetAsync(d->letters + d->total, 25, 64, ctx->stream));
    if (d->total)
      DRG_CUDA(cudaMemcpyAsync(d->letters, letters, d->total, cudaMemcpyHostToDevice, ctx->stream));
    DRG_CUDA(cudaMemcpyAsync(d->offsets, offsets, (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, ctx->stream));
    launch_letter_owner(d->offsets, n, 0, d->total, d->owner, ctx->stream);
    clamp_for_dp(ctx, d);
  } catch (...) {
    free_db(d);
    throw;
  }
  return d;
}

drg_batch* make_batch(drg_ctx* ctx, const uint8_t* letters, const uint64_t* offsets, const uint32_t* query,
                      const uint8_t* frame, uint64_t n, const uint32_t* request) {
  drg_batch* b = new drg_batch();
  b->ctx = ctx;
  b->n = n;
  b->h_offsets.assign(offsets, offsets + n + 1);
  b->total = offsets[n];
  b->query.resize(n);
  b->frame.resize(n);
  for (uint64_t i = 0; i < n; ++i) {
    b->query[i] = query ? query[i] : (uint32_t)i;
    b->frame[i] = frame ? frame[i] : 0;
    if (offsets[i + 1] < offsets[i]) {
      delete b;
      throw Error(DRG_ERR_INVALID, "target offsets must be non-decreasing");
    }
    b->max_len = std::max<uint32_t>(b->max_len, (uint32_t)(offsets[i + 1] - offsets[i]));
  }
  try {
    pool_alloc(ctx, &b->letters, b->total + 64);
    pool_alloc(ctx, &b->offsets, (n + 1) * sizeof(uint64_t));
    pool_alloc(ctx, &b->owner, (b->total + 1) * sizeof(uint32_t));
    DRG_CUDA(cudaMemsetAsync(b->letters + b->total, 25, 64, ctx->stream));
    if (b->total)
      DRG_CUDA(cudaMemcpyAsync(b->letters, letters, b->total, cudaMemcpyHostToDevice, ctx->stream));
    DRG_CUDA(cudaMemcpyAsync(b->offsets, offsets, (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, ctx->stream));
    launch_letter_owner(b->offsets, n, 0, b->total, b->owner, ctx->stream);
    // per-request join accounting; a batch of one request counts over the
    // whole batch, which is the plain search (narrower seed keys)
    bool several = false;
    for (uint64_t i = 0; request && i < n; ++i) {
      if (request[i] > kMaxRequests) throw Error(DRG_ERR_INVALID, "request id out of range");
      several = several || request[i] != request[0];
      b->max_request = std::max(b->max_request, request[i]);
    }
    if (several) {
      pool_alloc(ctx, &b->request, n * sizeof(uint32_t));
      DRG_CUDA(cudaMemcpyAsync(b->request, request, n * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
    }
    clamp_for_dp(ctx, b);
  } catch (...) {
    free_batch(b);
    throw;
  }
  return b;
}

drg_batch* make_batch_translated(drg_ctx* ctx, const uint8_t* nt, const uint64_t* nt_off, uint64_t n_reads,
                                 int64_t min_orf, HostFrames* host) {
  const uint64_t n_nt = nt_off[n_reads];
  for (uint64_t i = 0; i < n_reads; ++i)
    if (nt_off[i + 1] < nt_off[i]) throw Error(DRG_ERR_INVALID, "read offsets must be non-decreasing");
  if (6 * n_reads > 0xFFFFFFF0ull) throw Error(DRG_ERR_INVALID, "too many reads in one batch");
  drg_ctx* c = ctx;
  const uint64_t n6 = 6 * n_reads;
  uint8_t* d_nt = c->x_nt.as<uint8_t>(n_nt + 16);
  uint64_t* d_off = c->x_nt_off.as<uint64_t>(n_reads + 1);
  if (n_nt) DRG_CUDA(cudaMemcpyAsync(d_nt, nt, n_nt, cudaMemcpyHostToDevice, c->stream));
  DRG_CUDA(cudaMemcpyAsync(d_off, nt_off, (n_reads + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
  uint64_t* len = c->x_len.as<uint64_t>(n6 + 1);
  uint64_t* soff = c->x_scratch_off.as<uint64_t>(n6 + 1);
  launch_frame_lengths(d_off, n_reads, len, c->stream);
  cub_call(c, [&](void* t, size_t& b) {
    return cub::DeviceScan::ExclusiveSum(t, b, len, soff, (int64_t)n6 + 1, c->stream);
  });
  const uint64_t n_scratch = fetch(c, soff + n6);
  TranslateArgs a{};
  a.nt = d_nt;
  a.nt_off = d_off;
  a.n_reads = n_reads;
  a.min_orf = min_orf;
  a.scratch = c->x_scratch.as<uint8_t>(n_scratch + 16);
  a.scratch_off = soff;
  a.keep = c->x_keep.as<uint32_t>(n6 + 1);
  a.kept_len = c->x_kept_len.as<uint64_t>(n6 + 1);
  uint32_t* kidx = c->x_kept_index.as<uint32_t>(n6 + 1);
  uint64_t* koff = c->x_kept_off.as<uint64_t>(n6 + 1);
  a.kept_index = kidx;
  a.kept_off = koff;
  launch_translate_frames(a, c->stream);
  cub_call(c, [&](void* t, size_t& b) {
    return cub::DeviceScan::ExclusiveSum(t, b, a.keep, kidx, (int64_t)n6 + 1, c->stream);
  });
  cub_call(c, [&](void* t, size_t& b) {
    return cub::DeviceScan::ExclusiveSum(t, b, a.kept_len, koff, (int64_t)n6 + 1, c->stream);
  });
  const uint64_t n = fetch(c, kidx + n6);
  const uint64_t total = fetch(c, koff + n6);
  drg_batch* b = new drg_batch();
  b->ctx = ctx;
  b->n = n;
  b->total = total;
  try {
    pool_alloc(ctx, &b->letters, total + 64);
    pool_alloc(ctx, &b->offsets, (n + 1) * sizeof(uint64_t));
    pool_alloc(ctx, &b->owner, (total + 1) * sizeof(uint32_t));
    DRG_CUDA(cudaMemsetAsync(b->letters + total, 25, 64, ctx->stream));
    a.out = b->letters;
    a.out_off = b->offsets;
    a.out_query = c->x_query.as<uint32_t>(n + 1);
    a.out_frame = c->x_frame.as<uint8_t>(n + 1);
    launch_compact_frames(a, c->stream);
    launch_letter_owner(b->offsets, n, 0, total, b->owner, ctx->stream);
    fetch_n(c, b->h_offsets, b->offsets, n + 1);
    fetch_n(c, b->query, a.out_query, n);
    fetch_n(c, b->frame, a.out_frame, n);
    for (uint64_t i = 0; i < n; ++i)
      b->max_len = std::max<uint32_t>(b->max_len, (uint32_t)(b->h_offsets[i + 1] - b->h_offsets[i]));
    if (host) {
      fetch_n(c, host->letters, b->letters, total);
      host->offsets = b->h_offsets;
      host->query = b->query;
      host->frame = b->frame;
    }
  } catch (...) {
    free_batch(b);
    throw;
  }
  return b;
}

void free_db(drg_db* d) {
  if (!d) return;
  d->cache.reset();
  pool_free(d->ctx, d->letters);
  pool_free(d->ctx, d->score_letters);
  pool_free(d->ctx, d->offsets);
  pool_free(d->ctx, d->owner);
  delete d;
}

void free_batch(drg_batch* b) {
  if (!b) return;
  pool_free(b->ctx, b->letters);
  pool_free(b->ctx, b->score_letters);
  pool_free(b->ctx, b->offsets);
  pool_free(b->ctx, b->owner);
  pool_free(b->ctx, b->request);
  delete b;
}

}  // namespace drg
