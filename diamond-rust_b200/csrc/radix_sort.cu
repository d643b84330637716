// Device LSD radix sort (onesweep form) for the seed, hit, band and task keys.
//
// seed::build sorts its entries by key (seed.rs:102) and align_target sorts a
// subject's hits (search.rs:178); here every such sort is one LSD radix sort
// over the bits the keys use:
//
//   k_radix_hist    one pass over the keys (128-bit loads) counting every
//                   digit of every pass in shared memory
//   k_radix_scan    exclusive scan of each pass's 256 digit counts
//   k_onesweep      one persistent launch per 8-bit digit: a tile of 256
//                   threads x ITEMS keys is loaded with 128-bit loads through
//                   shared memory, ranked stably (per-warp __match_any_sync,
//                   then a scan over warps), its global position per digit
//                   found by decoupled look-back over the preceding tiles
//                   (words tagged with the pass's epoch, so the look-back
//                   area is never cleared between passes), and
//                   scattered through shared memory so that the stores of one
//                   digit run are contiguous.
//
// The element count is read from device memory, so a sort can follow the
// kernel that produced its input without a host round trip: the grid is at
// most the blocks that fit on the device at once, and each block takes tiles
// from an atomic counter until the count is covered.  Tiles are taken in the
// order blocks reach the counter, so a tile only ever waits on tiles that
// running blocks hold; each wait is bounded, and a wait that gives up sets an
// error word that the host checks (the outputs are then not used).
#include <algorithm>
#include <cstdint>

#include "kernels.h"

namespace drg {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kBins = 256;
// Look-back word: epoch (16 bits, the pass's tag) | status (2 bits:
// 1 aggregate, 2 inclusive) | count (46 bits).  A word of another epoch reads
// as "not ready", so the look-back area needs no clearing between passes.
constexpr uint64_t kAggregate = 1ull << 46, kInclusive = 2ull << 46, kCountMask = (1ull << 46) - 1;
__device__ __forceinline__ uint64_t lb_word(uint32_t epoch, uint64_t status, uint64_t count) {
  return ((uint64_t)epoch << 48) | status | (count & kCountMask);
}
constexpr int kSpinLimit = 1 << 22;

// Keys per thread of a tile: large tiles (16 u32 / 12 u64 keys per thread,
// 4,096 / 3,072 per tile) or small ones (half that: more tiles, a shorter
// wait per look-back step).  The context's tuning picks one.
template <typename K, bool SMALL>
struct SortItems;
template <>
struct SortItems<uint32_t, false> {
  static constexpr int value = 16;
};
template <>
struct SortItems<uint32_t, true> {
  static constexpr int value = 8;
};
template <>
struct SortItems<uint64_t, false> {
  static constexpr int value = 12;
};
template <>
struct SortItems<uint64_t, true> {
  static constexpr int value = 6;
};

__device__ __forceinline__ uint64_t sort_count(const uint64_t* d_n, uint64_t n_host) {
  return d_n ? *d_n : n_host;
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const K* __restrict__ keys, const uint64_t* d_n,
                                                             uint64_t n_host, int begin_bit, int end_bit, int passes,
                                                             int dbits, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[8][kBins];
  for (int i = threadIdx.x; i < 8 * kBins; i += kSortThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  const uint64_t n = sort_count(d_n, n_host);
  auto add = [&](K k) {
    for (int p = 0; p < passes; ++p) {
      const int sh = begin_bit + p * dbits;
      const int db = end_bit - sh < dbits ? end_bit - sh : dbits;  // the last digit may be narrower
      atomicAdd(&h[p][(uint32_t)(k >> sh) & ((1u << db) - 1)], 1u);
    }
  };
  constexpr int kPer = 16 / sizeof(K);
  const bool vec = (reinterpret_cast<uintptr_t>(keys) & 15) == 0;
  const uint64_t n_vec = vec ? n / kPer : 0;
  const uint64_t stride = (uint64_t)gridDim.x * kSortThreads;
  for (uint64_t v = blockIdx.x * (uint64_t)kSortThreads + threadIdx.x; v < n_vec; v += stride) {
    const uint4 q = reinterpret_cast<const uint4*>(keys)[v];
    const K* e = reinterpret_cast<const K*>(&q);
#pragma unroll
    for (int j = 0; j < kPer; ++j) add(e[j]);
  }
  for (uint64_t i = n_vec * kPer + blockIdx.x * (uint64_t)kSortThreads + threadIdx.x; i < n; i += stride) add(keys[i]);
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kBins; i += kSortThreads) {
    const uint32_t c = (&h[0][0])[i];
    if (c) atomicAdd(&hist[i], c);
  }
}

// Exclusive scan of each pass's digit counts (one block per pass).
__global__ void __launch_bounds__(kBins) k_radix_scan(const uint32_t* __restrict__ hist, uint32_t* __restrict__ start) {
  __shared__ uint32_t warp_tot[kBins / 32];
  const int p = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5;
  const uint32_t c = hist[p * kBins + t];
  uint32_t x = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  uint32_t base = 0;
  for (int i = 0; i < w; ++i) base += warp_tot[i];
  start[p * kBins + t] = base + x - c;
}

template <typename K, bool VALS, bool SMALL>
struct alignas(16) OnesweepShared {
  static constexpr int kItems = SortItems<K, SMALL>::value;
  static constexpr int kTile = kSortThreads * kItems;
  union {
    K keys[kTile];
    uint32_t vals[kTile];
  } stage;
  uint32_t warp_cnt[kSortWarps][kBins];
  uint8_t digit[kTile];
  uint32_t global_base[kBins];  // out index of tile-local position 0 of each digit
  uint32_t scan_tot[kSortWarps];
  uint32_t tile;
};

// Loads tile keys [0, valid) into sh (128-bit loads where aligned).
template <typename K>
__device__ __forceinline__ void load_tile(const K* __restrict__ src, uint64_t base, int valid, K* sh) {
  constexpr int kPer = 16 / sizeof(K);
  const K* p = src + base;
  if ((reinterpret_cast<uintptr_t>(p) & 15) == 0) {
    const int nv = valid / kPer;
    for (int v = threadIdx.x; v < nv; v += kSortThreads)
      reinterpret_cast<uint4*>(sh)[v] = reinterpret_cast<const uint4*>(p)[v];
    for (int i = nv * kPer + threadIdx.x; i < valid; i += kSortThreads) sh[i] = p[i];
  } else {
    for (int i = threadIdx.x; i < valid; i += kSortThreads) sh[i] = p[i];
  }
}

// One tile of one digit pass (s.warp_cnt zeroed, tile < tiles of the count).
template <typename K, bool VALS, bool SMALL>
__device__ __forceinline__ void onesweep_tile(OnesweepShared<K, VALS, SMALL>& s, uint32_t tile, uint64_t n,
                                              const K* __restrict__ kin, K* __restrict__ kout,
                                              const uint32_t* __restrict__ vin, uint32_t* __restrict__ vout,
                                              int shift, int dbits, const uint32_t* __restrict__ digit_start,
                                              uint64_t* lookback, uint32_t epoch, uint32_t* err) {
  using Sh = OnesweepShared<K, VALS, SMALL>;
  constexpr int kItems = Sh::kItems, kTile = Sh::kTile;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const uint64_t base = (uint64_t)tile * kTile;
  const int valid = n - base < (uint64_t)kTile ? (int)(n - base) : kTile;
  const uint32_t mask = (1u << dbits) - 1;

  // ---- keys: coalesced 128-bit loads into shared memory, then warp-striped
  // registers (item j of lane l in warp w is tile element w*32*ITEMS + j*32 + l,
  // so processing items in j order, lanes within, is input order)
  load_tile(kin, base, valid, s.stage.keys);
  __syncthreads();
  K key[kItems];
  uint32_t dig[kItems];
  uint16_t pos[kItems];
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const int e = w * 32 * kItems + j * 32 + lane;
    key[j] = e < valid ? s.stage.keys[e] : (K)0;
    // past the end: the largest digit value, so such items rank after every
    // real item of the tile (they are last in input order)
    dig[j] = e < valid ? (uint32_t)(key[j] >> shift) & mask : (uint32_t)(kBins - 1);
  }
  // ---- stable rank within the warp
  const uint32_t lt = (1u << lane) - 1;
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, dig[j]);
    const uint32_t before = s.warp_cnt[w][dig[j]];
    __syncwarp();
    if ((peers & lt) == 0) s.warp_cnt[w][dig[j]] = before + __popc(peers);
    __syncwarp();
    pos[j] = (uint16_t)(before + __popc(peers & lt));
  }
  __syncthreads();
  // ---- tile-local digit starts: thread t owns digit t
  uint32_t run = 0;
#pragma unroll
  for (int i = 0; i < kSortWarps; ++i) {
    const uint32_t c = s.warp_cnt[i][t];
    s.warp_cnt[i][t] = run;
    run += c;
  }
  const uint32_t count = run;
  uint32_t x = count;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s.scan_tot[w] = x;
  __syncthreads();
  uint32_t local_start = x - count;
  for (int i = 0; i < w; ++i) local_start += s.scan_tot[i];
#pragma unroll
  for (int i = 0; i < kSortWarps; ++i) s.warp_cnt[i][t] += local_start;
  // ---- decoupled look-back: this tile's count of digit t, and the counts of
  // the tiles before it
  const uint32_t mine = count - (t == kBins - 1 ? (uint32_t)(kTile - valid) : 0u);
  volatile uint64_t* lb = lookback;
  uint32_t excl = 0;
  if (tile == 0) {
    lb[t] = lb_word(epoch, kInclusive, mine);
  } else {
    lb[(uint64_t)tile * kBins + t] = lb_word(epoch, kAggregate, mine);
    for (int64_t p = (int64_t)tile - 1; p >= 0; --p) {
      uint64_t v;
      int it = 0;
      while (((v = lb[(uint64_t)p * kBins + t]) >> 48) != epoch || (v & ~kCountMask & ((1ull << 48) - 1)) == 0) {
        if (++it > kSpinLimit) {
          atomicOr(err, 1u);
          v = lb_word(epoch, kInclusive, 0);
          break;
        }
        if (it > 64) __nanosleep(64);
      }
      excl += (uint32_t)(v & kCountMask);
      if ((v & kInclusive) != 0) break;
    }
    lb[(uint64_t)tile * kBins + t] = lb_word(epoch, kInclusive, excl + mine);
  }
  s.global_base[t] = digit_start[t] + excl - local_start;
  __syncthreads();
  // ---- keys to their tile-local sorted place, then out in digit runs
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const uint32_t p = s.warp_cnt[w][dig[j]] + pos[j];
    pos[j] = (uint16_t)p;
    s.stage.keys[p] = key[j];
    s.digit[p] = (uint8_t)dig[j];
  }
  __syncthreads();
  // (32-bit arithmetic: global_base may be "negative"; every position is
  // below n < 2^32, so the sum modulo 2^32 is the position)
  for (int i = t; i < valid; i += kSortThreads) {
    const uint32_t o = s.global_base[s.digit[i]] + (uint32_t)i;
    if (o < n) kout[o] = s.stage.keys[i];
  }
  if (!VALS) return;
  __syncthreads();
  // ---- values: the same permutation
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const int e = w * 32 * kItems + j * 32 + lane;
    if (e < valid) s.stage.vals[pos[j]] = vin[base + e];
  }
  __syncthreads();
  for (int i = t; i < valid; i += kSortThreads) {
    const uint32_t o = s.global_base[s.digit[i]] + (uint32_t)i;
    if (o < n) vout[o] = s.stage.vals[i];
  }
}

// A persistent grid (at most the blocks that fit on the device at once):
// each block takes tiles from the pass's counter until they run out.
template <typename K, bool VALS, bool SMALL>
__global__ void __launch_bounds__(kSortThreads, 3) k_onesweep(const K* __restrict__ kin, K* __restrict__ kout,
                                                              const uint32_t* __restrict__ vin,
                                                              uint32_t* __restrict__ vout, const uint64_t* d_n,
                                                              uint64_t n_host, int shift, int dbits,
                                                              const uint32_t* __restrict__ digit_start,
                                                              uint64_t* lookback, uint32_t epoch,
                                                              uint32_t* tile_counter, uint32_t* err) {
  using Sh = OnesweepShared<K, VALS, SMALL>;
  __shared__ Sh s;
  const uint64_t n = sort_count(d_n, n_host);
  for (;;) {
    if (threadIdx.x == 0) s.tile = atomicAdd(tile_counter, 1u);
    for (int i = threadIdx.x; i < kSortWarps * kBins; i += kSortThreads) (&s.warp_cnt[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = s.tile;
    if ((uint64_t)tile * Sh::kTile >= n) return;  // every thread sees the same tile
    onesweep_tile<K, VALS, SMALL>(s, tile, n, kin, kout, vin, vout, shift, dbits, digit_start, lookback, epoch,
                                  err);
    __syncthreads();  // the next tile reuses the shared state
  }
}

// Blocks of k_onesweep<K, VALS, SMALL> that fit on the current device at once.
template <typename K, bool VALS, bool SMALL>
int onesweep_resident_blocks() {
  static int cached[64] = {};
  int dev = 0;
  DRG_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && cached[dev]) return cached[dev];
  int per_sm = 0, sms = 0;
  DRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_onesweep<K, VALS, SMALL>, kSortThreads, 0));
  DRG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int r = std::max(1, per_sm) * std::max(1, sms);
  if (dev >= 0 && dev < 64) cached[dev] = r;
  return r;
}

constexpr int kMaxPasses = 8;  // 64-bit keys in 8-bit digits

struct SortPlan {
  int passes = 0, dbits = 8;
  uint64_t tiles = 0;
  size_t hist_off = 0, start_off = 0, ctr_off = 0, lb_off = 0, bytes = 0;
};

template <typename K>
SortPlan plan(uint64_t n_max, int begin_bit, int end_bit, bool small) {
  SortPlan p;
  const int bits = end_bit - begin_bit;
  if (bits <= 0) return p;
  p.passes = (bits + 7) / 8;
  p.dbits = (bits + p.passes - 1) / p.passes;  // digit width per pass
  const uint64_t tile =
      (uint64_t)kSortThreads * (small ? SortItems<K, true>::value : SortItems<K, false>::value);
  p.tiles = n_max == 0 ? 1 : (n_max + tile - 1) / tile;
  // Histograms, digit starts and tile counters are laid out for the most
  // passes any sort takes, so that the look-back area starts at the same
  // offset in every sort and holds nothing but look-back words (or zeros).
  p.hist_off = 0;
  p.start_off = p.hist_off + (size_t)kMaxPasses * kBins * 4;
  p.ctr_off = p.start_off + (size_t)kMaxPasses * kBins * 4;
  p.lb_off = (p.ctr_off + kMaxPasses * 4 + 255) & ~size_t(255);
  p.bytes = p.lb_off + (size_t)p.tiles * kBins * 8;  // one look-back area, reused by every pass (epochs)
  return p;
}

}  // namespace

template <typename K>
SortResult<K> radix_sort(K* keys, K* keys_alt, uint32_t* vals, uint32_t* vals_alt, uint64_t n_max,
                         const uint64_t* d_n, int begin_bit, int end_bit, SortScratch& temp, uint32_t* d_err,
                         cudaStream_t st, bool small_tiles) {
  SortResult<K> r{keys, vals};
  if (n_max >= (1ull << 32)) throw Error(DRG_ERR_INVALID, "radix sort: at most 2^32 - 1 keys per sort");
  if (end_bit > (int)(8 * sizeof(K))) end_bit = 8 * sizeof(K);
  const SortPlan p = plan<K>(n_max, begin_bit, end_bit, small_tiles);
  if (p.passes == 0 || (n_max == 0 && !d_n)) return r;
  // (a reallocation shows in the capacity: the new block may start at the
  // old address, holding another buffer's stale words)
  const size_t cap_before = temp.buf.cap;
  uint8_t* tb = static_cast<uint8_t*>(temp.buf.ensure(p.bytes));
  uint32_t* hist = reinterpret_cast<uint32_t*>(tb + p.hist_off);
  uint32_t* start = reinterpret_cast<uint32_t*>(tb + p.start_off);
  uint32_t* ctr = reinterpret_cast<uint32_t*>(tb + p.ctr_off);
  uint64_t* lb = reinterpret_cast<uint64_t*>(tb + p.lb_off);
  // new memory, or epochs about to wrap: clear the look-back area once
  if (temp.buf.cap != cap_before || temp.epoch + (uint32_t)p.passes >= 0xFFFFu) {
    DRG_CUDA(cudaMemsetAsync(tb, 0, temp.buf.cap, st));
    temp.epoch = 0;
  }
  DRG_CUDA(cudaMemsetAsync(tb, 0, p.lb_off, st));  // histograms, digit starts, tile counters
  const int hist_blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((n_max + 4095) / 4096, 148 * 4));
  count_launch();
  k_radix_hist<K><<<hist_blocks, kSortThreads, 0, st>>>(keys, d_n, n_max, begin_bit, end_bit, p.passes, p.dbits,
                                                         hist);
  DRG_CUDA(cudaGetLastError());
  count_launch();
  k_radix_scan<<<p.passes, kBins, 0, st>>>(hist, start);
  DRG_CUDA(cudaGetLastError());
  K *ki = keys, *ko = keys_alt;
  uint32_t *vi = vals, *vo = vals_alt;
  for (int pass = 0; pass < p.passes; ++pass) {
    const int shift = begin_bit + pass * p.dbits;
    const int db = std::min(p.dbits, end_bit - shift);
    count_launch();
    const uint32_t epoch = ++temp.epoch;  // 1..65534
    auto launch = [&](auto kernel, int resident) {
      const unsigned grid = (unsigned)std::min<uint64_t>(p.tiles, (uint64_t)resident);
      kernel<<<grid, kSortThreads, 0, st>>>(ki, ko, vi, vo, d_n, n_max, shift, db, start + pass * kBins, lb, epoch,
                                            ctr + pass, d_err);
    };
    if (vals && small_tiles)
      launch(k_onesweep<K, true, true>, onesweep_resident_blocks<K, true, true>());
    else if (vals)
      launch(k_onesweep<K, true, false>, onesweep_resident_blocks<K, true, false>());
    else if (small_tiles)
      launch(k_onesweep<K, false, true>, onesweep_resident_blocks<K, false, true>());
    else
      launch(k_onesweep<K, false, false>, onesweep_resident_blocks<K, false, false>());
    DRG_CUDA(cudaGetLastError());
    std::swap(ki, ko);
    std::swap(vi, vo);
  }
  r.keys = ki;
  r.vals = vals ? vi : nullptr;
  return r;
}

template SortResult<uint32_t> radix_sort<uint32_t>(uint32_t*, uint32_t*, uint32_t*, uint32_t*, uint64_t,
                                                   const uint64_t*, int, int, SortScratch&, uint32_t*, cudaStream_t,
                                                   bool);
template SortResult<uint64_t> radix_sort<uint64_t>(uint64_t*, uint64_t*, uint32_t*, uint32_t*, uint64_t,
                                                   const uint64_t*, int, int, SortScratch&, uint32_t*, cudaStream_t,
                                                   bool);

}  // namespace drg
