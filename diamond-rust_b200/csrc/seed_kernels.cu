// Seed enumeration (shape.rs:60-75, seed.rs:46-104) and the sort-merge
// double-index join (seed.rs:110-143) on the device.
//
// Layout: one thread per letter, looping over the shapes, so that a warp
// reads each shape's table entries at one constant address (a broadcast) and
// writes each shape's keys as one coalesced run: entry s * L + i holds shape
// s at letter i.  Letters of a sequence batch are contiguous in HBM, so the w
// reads of a seed hit one or two 32-byte sectors shared by neighbouring
// threads.  Seeds are written as 64-bit keys (request | shape | key) with a
// 32-bit payload (the global letter index) and sorted by the device radix
// sort (stable: equal keys share a shape and stay in letter order, as in the
// reference's build); the join walks query key runs and binary-searches the
// sorted reference keys.
#include <cmath>

#include "kernels.h"

namespace drg {

// One bank per context slot, so that contexts searching with different
// presets at the same time do not overwrite each other's tables.
__constant__ ShapeTable c_shapes[kConstSlots];
__constant__ SeedParams c_seed[kConstSlots];

// The complexity test (seed.rs:58-75) keeps a seed of weight w when
// e = ln w! - sum over buckets of ln c_b! >= cut, that is when the integer
// P = prod c_b! is at most T_w = exp(ln w! - cut).  P decides outright when it
// lies outside T_w (1 -+ 1e-7): e then differs from the cut by more than
// 1e-7, far above the 1e-13 rounding of the reference's double sum.  Closer
// to T_w the device evaluates that sum in the reference's order.
void seed_cut_bounds(SeedParams& p) {
  for (int w = 0; w <= kMaxWeight; ++w) {
    if (!(p.cut > 0.0)) {
      p.p_accept[w] = UINT64_MAX;
      p.p_reject[w] = UINT64_MAX;
      continue;
    }
    const double t = std::exp(p.lnfact[w] - p.cut);
    const double lo = t * (1.0 - 1e-7), hi = t * (1.0 + 1e-7);
    p.p_accept[w] = lo < 1.0 ? 0 : (lo >= 1.8e19 ? UINT64_MAX : (uint64_t)std::floor(lo));
    p.p_reject[w] = hi >= 1.8e19 ? UINT64_MAX : (uint64_t)std::ceil(hi);
  }
}

void upload_seed_params(const ShapeTable& shapes, const SeedParams& params, int slot, cudaStream_t st) {
  SeedParams p = params;
  seed_cut_bounds(p);
  p.key32 = 1;
  p.prod32 = 1;
  for (int s = 0; s < shapes.n; ++s) {
    double mx = 1.0;
    for (int k = 0; k < shapes.weight[s]; ++k) mx *= (double)p.size;
    if (mx > 4294967295.0) p.key32 = 0;
    if (shapes.weight[s] > 12) p.prod32 = 0;
  }
  DRG_CUDA(cudaMemcpyToSymbolAsync(c_shapes, &shapes, sizeof(ShapeTable), slot * sizeof(ShapeTable),
                                   cudaMemcpyHostToDevice, st));
  DRG_CUDA(cudaMemcpyToSymbolAsync(c_seed, &p, sizeof(SeedParams), slot * sizeof(SeedParams),
                                   cudaMemcpyHostToDevice, st));  // pageable source: staged before return
}

__global__ void k_letter_owner(const uint64_t* __restrict__ offsets, uint64_t n_seqs, uint64_t lo, uint64_t hi,
                               uint32_t* __restrict__ out) {
  uint64_t g = lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (g >= hi) return;
  // largest i with offsets[i] <= g (sequences may be empty)
  uint64_t a = 0, b = n_seqs;  // answer in [a, b)
  while (b - a > 1) {
    uint64_t m = (a + b) >> 1;
    if (offsets[m] <= g) a = m;
    else b = m;
  }
  out[g - lo] = (uint32_t)a;
}

// Letter codes above 24 score as 24 (matrix.rs:164-168 clamps both indices)
// but would index past the packed kernels' 26-row residue profiles: any such
// byte sets *bad, and the DP kernels then read a clamped copy.  Sixteen
// letters per thread (the buffers are 256-byte aligned), four at a time.
__global__ void k_check_letters(const uint8_t* __restrict__ letters, uint64_t n, unsigned int* __restrict__ bad) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  bool b = false;
  if (16 * t + 16 <= n) {
    const uint4 w = reinterpret_cast<const uint4*>(letters)[t];
    b = (__vcmpgtu4(w.x, 0x18181818u) | __vcmpgtu4(w.y, 0x18181818u) | __vcmpgtu4(w.z, 0x18181818u) |
         __vcmpgtu4(w.w, 0x18181818u)) != 0;
  } else {
    for (uint64_t i = 16 * t; i < n; ++i) b |= letters[i] > 24;
  }
  if (__any_sync(0xFFFFFFFFu, b) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
}

__global__ void k_clamp_letters(const uint8_t* __restrict__ in, uint64_t n, uint8_t* __restrict__ out) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i] < 24 ? in[i] : 24;
}

void launch_clamp_letters(const uint8_t* in, uint64_t n, uint8_t* out, cudaStream_t st) {
  if (n == 0) return;
  count_launch();
  k_clamp_letters<<<ceil_div((long long)n, 256), 256, 0, st>>>(in, n, out);
  DRG_CUDA(cudaGetLastError());
}

void launch_check_letters(const uint8_t* letters, uint64_t n, unsigned int* bad, cudaStream_t st) {
  DRG_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned int), st));
  if (n == 0) return;
  count_launch();
  k_check_letters<<<ceil_div(ceil_div((long long)n, 16), 256), 256, 0, st>>>(letters, n, bad);
  DRG_CUDA(cudaGetLastError());
}

void launch_letter_owner(const uint64_t* offsets, uint64_t n_seqs, uint64_t lo, uint64_t hi, uint32_t* out,
                         cudaStream_t st) {
  if (hi <= lo || n_seqs == 0) return;
  count_launch();
  k_letter_owner<<<ceil_div(hi - lo, 256), 256, 0, st>>>(offsets, n_seqs, lo, hi, out);
  DRG_CUDA(cudaGetLastError());
}

// Seed enumeration runs one thread per letter in blocks of kEnumBlock; each
// block first turns its letters (plus the longest span past the last one)
// into reduced buckets in shared memory, 255 for a letter that cannot seed
// (a code of 20 or more, a letter outside the reduction, or past the range).
constexpr int kEnumBlock = 256;

struct EnumTables {
  uint8_t rb[kEnumBlock + kMaxSpan];
};

__device__ __forceinline__ void stage_enum_tables(const uint8_t* __restrict__ letters, uint64_t base, uint64_t hi,
                                                  int slot, EnumTables& t) {
  const SeedParams& sp = c_seed[slot];
  for (int j = threadIdx.x; j < kEnumBlock + kMaxSpan; j += blockDim.x) {
    const uint64_t g = base + j;
    uint8_t b = 255;
    if (g < hi) {
      const uint32_t l = letters[g];
      if (l < 20) b = sp.bucket[l];
    }
    t.rb[j] = b;
  }
  __syncthreads();
}

// One seed from the staged buckets at rb: the reduced key and the
// complexity test (seed.rs).  Bucket counts live in 5-bit fields of two
// words (buckets 0-11 and 12-23), updated without branches; P collects the
// count after each letter, so that P = prod over buckets of c_b!.  KT holds
// the key (32 bits when size^w fits), PT the product (32 bits when w <= 12).
template <typename KT, typename PT>
__device__ __forceinline__ bool seed_at_t(const uint8_t* rb, int s, int slot, uint64_t* key_out) {
  const ShapeTable& shp = c_shapes[slot];
  const SeedParams& sp = c_seed[slot];
  const int w = shp.weight[s];
  const KT size = (KT)sp.size;
  KT key = 0;
  uint64_t lo = 0, hi = 0;
  PT prod = 1;
  for (int k = 0; k < w; ++k) {
    const uint32_t b = rb[shp.pos[s][k]];
    if (b >= 24) return false;
    key = key * size + (KT)b;
    const bool up = b >= 12;
    const uint32_t sh = 5 * (up ? b - 12 : b);
    const uint64_t inc = 1ull << sh;
    lo += up ? 0ull : inc;
    hi += up ? inc : 0ull;
    prod *= (PT)(((up ? hi : lo) >> sh) & 31u);
  }
  if (sp.cut > 0.0) {
    const uint64_t P = (uint64_t)prod;
    if (P > sp.p_accept[w]) {
      if (P >= sp.p_reject[w]) return false;
      // within 1e-7 of the cut: ln w! minus ln c_b! in bucket order, as the
      // reference sums it
      double e = sp.lnfact[w];
      for (int b = 0; b < (int)sp.size; ++b) {
        const uint32_t c = (uint32_t)(((b < 12 ? lo : hi) >> (5 * (b < 12 ? b : b - 12))) & 31u);
        if (c > 0) e = __dsub_rn(e, sp.lnfact[c]);
      }
      if (!(e >= sp.cut)) return false;
    }
  }
  *key_out = (uint64_t)key;
  return true;
}

__device__ __forceinline__ bool seed_at(const uint8_t* rb, int s, int slot, uint64_t* key_out) {
  const SeedParams& sp = c_seed[slot];
  if (sp.key32 && sp.prod32) return seed_at_t<uint32_t, uint32_t>(rb, s, slot, key_out);
  return seed_at_t<uint64_t, uint64_t>(rb, s, slot, key_out);
}

// Hash of a seed key (shape | key) into a bitmap of 2^log2_bits bits.
__device__ __forceinline__ uint32_t seed_key_hash(uint64_t k, int log2_bits) {
  return (uint32_t)((k * 0x9E3779B97F4A7C15ull) >> (64 - log2_bits));  // Fibonacci hashing
}

// K = uint32_t: the caller guarantees that the seed key (with the request,
// if any) fits 32 bits; "no seed" is then 0xFFFFFFFF.
// filter (optional): the bit of every valid seed's key (without the request)
// is set in it, the query-key bitmap of the filtered reference enumeration.
template <typename K>
__global__ void k_seed_enum(const uint8_t* __restrict__ letters, const uint64_t* __restrict__ offsets,
                            const uint32_t* __restrict__ owner, uint64_t lo, uint64_t hi, int n_shapes,
                            K* __restrict__ keys, uint32_t* __restrict__ vals,
                            const uint32_t* __restrict__ request, int slot, uint32_t* __restrict__ filter = nullptr,
                            int filter_log2 = 0) {
  __shared__ EnumTables tab;
  const uint64_t L = hi - lo;
  const uint64_t i = blockIdx.x * (uint64_t)kEnumBlock + threadIdx.x;
  stage_enum_tables(letters, lo + blockIdx.x * (uint64_t)kEnumBlock, hi, slot, tab);
  if (i >= L) return;
  const uint64_t g = lo + i;
  const uint32_t seq = owner[i];
  const uint64_t end = offsets[seq + 1];
  const SeedParams& sp = c_seed[slot];
  const uint64_t req = request ? (uint64_t)request[seq] << sp.request_shift : 0;
  for (int s = 0; s < n_shapes; ++s) {
    uint64_t key = 0;
    const bool ok = g + c_shapes[slot].span[s] <= end && seed_at(tab.rb + threadIdx.x, s, slot, &key);
    keys[s * L + i] = ok ? (K)(req | ((uint64_t)s << sp.shape_shift) | key) : (K)kNoSeed;
    vals[s * L + i] = (uint32_t)g;
    if (filter && ok) {
      const uint32_t h = seed_key_hash(((uint64_t)s << sp.shape_shift) | key, filter_log2);
      const uint32_t bit = 1u << (h & 31);
      if (!(filter[h >> 5] & bit)) atomicOr(filter + (h >> 5), bit);
    }
  }
}

void launch_seed_enum(const uint8_t* letters, const uint64_t* offsets, const uint32_t* owner, uint64_t lo,
                      uint64_t hi, int n_shapes, uint64_t* keys, uint32_t* vals, int slot, cudaStream_t st,
                      const uint32_t* request) {
  if (hi <= lo || n_shapes == 0) return;
  count_launch();
  k_seed_enum<uint64_t><<<ceil_div(hi - lo, kEnumBlock), kEnumBlock, 0, st>>>(letters, offsets, owner, lo, hi,
                                                                             n_shapes, keys, vals, request, slot);
  DRG_CUDA(cudaGetLastError());
}

void launch_seed_enum(const uint8_t* letters, const uint64_t* offsets, const uint32_t* owner, uint64_t lo,
                      uint64_t hi, int n_shapes, uint32_t* keys, uint32_t* vals, int slot, cudaStream_t st,
                      uint32_t* filter, int filter_log2) {
  if (hi <= lo || n_shapes == 0) return;
  count_launch();
  k_seed_enum<uint32_t><<<ceil_div(hi - lo, kEnumBlock), kEnumBlock, 0, st>>>(
      letters, offsets, owner, lo, hi, n_shapes, keys, vals, nullptr, slot, filter, filter_log2);
  DRG_CUDA(cudaGetLastError());
}

// ---- reference seeds restricted to the query's seed keys --------------------
// A reference seed joins only query seeds with the same key, so a chunk's
// enumeration can keep just the seeds whose key has its bit set in a bitmap
// of the query keys.  The bitmap is hashed: a false positive only keeps a
// seed that then matches no query run, and no key of the query is missed.


__global__ void k_key_filter(const uint64_t* __restrict__ run_keys, uint64_t n, uint64_t key_mask,
                             uint32_t* __restrict__ filter, int log2_bits) {
  const uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (u >= n) return;
  const uint32_t h = seed_key_hash(run_keys[u] & key_mask, log2_bits);
  const uint32_t bit = 1u << (h & 31);
  if (!(filter[h >> 5] & bit)) atomicOr(filter + (h >> 5), bit);
}

void launch_key_filter(const uint64_t* run_keys, uint64_t n, uint64_t key_mask, uint32_t* filter, int log2_bits,
                       cudaStream_t st) {
  if (n == 0) return;
  count_launch();
  k_key_filter<<<ceil_div(n, 256), 256, 0, st>>>(run_keys, n, key_mask, filter, log2_bits);
  DRG_CUDA(cudaGetLastError());
}

// One thread per letter as in k_seed_enum.  Kept seeds collect in shared
// memory, kFilterGroup shapes at a time, and each block reserves its output
// range with one atomic per group; counts[0] = seeds kept, counts[1] = valid
// seeds (kept or not).  The output order depends on the blocks' timing; the
// caller sorts by key, and the hits made from them are sorted in full later.
constexpr int kFilterBlock = kEnumBlock, kFilterGroup = 8;

template <typename K>
__global__ void __launch_bounds__(kFilterBlock)
    k_seed_enum_filtered(const uint8_t* __restrict__ letters, const uint64_t* __restrict__ offsets,
                         const uint32_t* __restrict__ owner, uint64_t lo, uint64_t hi, int n_shapes,
                         const uint32_t* __restrict__ filter, int log2_bits, K* __restrict__ keys,
                         uint32_t* __restrict__ vals, unsigned long long* __restrict__ counts, int slot) {
  __shared__ EnumTables tab;
  __shared__ K s_keys[kFilterBlock * kFilterGroup];
  __shared__ uint32_t s_vals[kFilterBlock * kFilterGroup];
  __shared__ uint32_t s_n;
  __shared__ unsigned long long s_base, s_valid;
  if (threadIdx.x == 0) {
    s_n = 0;
    s_valid = 0;
  }
  stage_enum_tables(letters, lo + blockIdx.x * (uint64_t)kFilterBlock, hi, slot, tab);  // ends with a barrier
  const uint64_t L = hi - lo;
  const uint64_t i = blockIdx.x * (uint64_t)kFilterBlock + threadIdx.x;
  const bool in = i < L;
  const uint64_t g = lo + i;
  const uint64_t end = in ? offsets[owner[i] + 1] : 0;
  const SeedParams& sp = c_seed[slot];
  unsigned long long valid = 0;
  for (int s0 = 0; s0 < n_shapes; s0 += kFilterGroup) {
    const int s1 = min(n_shapes, s0 + kFilterGroup);
    for (int s = s0; s < s1; ++s) {
      uint64_t key = 0;
      if (in && g + c_shapes[slot].span[s] <= end && seed_at(tab.rb + threadIdx.x, s, slot, &key)) {
        ++valid;
        const uint64_t k = ((uint64_t)s << sp.shape_shift) | key;
        const uint32_t h = seed_key_hash(k, log2_bits);
        if (__ldg(filter + (h >> 5)) & (1u << (h & 31))) {
          const uint32_t e = atomicAdd(&s_n, 1u);
          s_keys[e] = (K)k;
          s_vals[e] = (uint32_t)g;
        }
      }
    }
    __syncthreads();
    const uint32_t n = s_n;
    if (threadIdx.x == 0 && n > 0) s_base = atomicAdd(counts, (unsigned long long)n);
    __syncthreads();  // every thread has read s_n and can see s_base
    const unsigned long long base = s_base;
    if (threadIdx.x == 0) s_n = 0;
    for (uint32_t e = threadIdx.x; e < n; e += kFilterBlock) {
      keys[base + e] = s_keys[e];
      vals[base + e] = s_vals[e];
    }
    __syncthreads();  // the buffer is free for the next group
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) valid += __shfl_xor_sync(0xFFFFFFFFu, valid, o);
  if ((threadIdx.x & 31) == 0 && valid) atomicAdd(&s_valid, valid);
  __syncthreads();
  if (threadIdx.x == 0 && s_valid) atomicAdd(counts + 1, s_valid);
}

template <typename K>
void seed_enum_filtered(const uint8_t* letters, const uint64_t* offsets, const uint32_t* owner, uint64_t lo,
                        uint64_t hi, int n_shapes, const uint32_t* filter, int log2_bits, K* keys, uint32_t* vals,
                        unsigned long long* counts, int slot, cudaStream_t st) {
  if (hi <= lo || n_shapes == 0) return;
  count_launch();
  k_seed_enum_filtered<K><<<ceil_div(hi - lo, kFilterBlock), kFilterBlock, 0, st>>>(
      letters, offsets, owner, lo, hi, n_shapes, filter, log2_bits, keys, vals, counts, slot);
  DRG_CUDA(cudaGetLastError());
}

void launch_seed_enum_filtered(const uint8_t* letters, const uint64_t* offsets, const uint32_t* owner, uint64_t lo,
                               uint64_t hi, int n_shapes, const uint32_t* filter, int log2_bits, uint64_t* keys,
                               uint32_t* vals, unsigned long long* counts, int slot, cudaStream_t st) {
  seed_enum_filtered(letters, offsets, owner, lo, hi, n_shapes, filter, log2_bits, keys, vals, counts, slot, st);
}

void launch_seed_enum_filtered(const uint8_t* letters, const uint64_t* offsets, const uint32_t* owner, uint64_t lo,
                               uint64_t hi, int n_shapes, const uint32_t* filter, int log2_bits, uint32_t* keys,
                               uint32_t* vals, unsigned long long* counts, int slot, cudaStream_t st) {
  seed_enum_filtered(letters, offsets, owner, lo, hi, n_shapes, filter, log2_bits, keys, vals, counts, slot, st);
}

// first[b] = the first of n sorted keys with key >> shift >= b, for b in
// [0, nb]; the join then searches one bucket's range instead of all keys.
template <typename K>
__global__ void k_bucket_first(const K* __restrict__ keys, uint64_t n, int shift, uint32_t nb,
                               uint32_t* __restrict__ first, const uint64_t* d_n) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > nb) return;
  if (d_n) n = *d_n;
  const uint64_t key = (uint64_t)b << shift;
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t m = (lo + hi) >> 1;
    if ((uint64_t)keys[m] < key) lo = m + 1;
    else hi = m;
  }
  first[b] = b == nb ? (uint32_t)n : (uint32_t)lo;
}

template <typename K>
void bucket_first(const K* keys, uint64_t n, int shift, uint32_t nb, uint32_t* first, cudaStream_t st,
                  const uint64_t* d_n) {
  count_launch();
  k_bucket_first<K><<<ceil_div((long long)nb + 1, 256), 256, 0, st>>>(keys, n, shift, nb, first, d_n);
  DRG_CUDA(cudaGetLastError());
}

void launch_bucket_first(const uint64_t* keys, uint64_t n, int shift, uint32_t nb, uint32_t* first, cudaStream_t st,
                         const uint64_t* d_n) {
  bucket_first(keys, n, shift, nb, first, st, d_n);
}

void launch_bucket_first(const uint32_t* keys, uint64_t n, int shift, uint32_t nb, uint32_t* first, cudaStream_t st,
                         const uint64_t* d_n) {
  bucket_first(keys, n, shift, nb, first, st, d_n);
}

template <typename K>
__global__ void k_join_count(const uint64_t* __restrict__ run_keys, const uint32_t* __restrict__ run_counts,
                             uint64_t n_runs, const K* __restrict__ ref_keys, uint64_t n_ref,
                             uint64_t max_expand, uint32_t* __restrict__ run_rlo, uint32_t* __restrict__ run_rcount,
                             uint64_t* __restrict__ run_hits, uint64_t key_mask, const uint32_t* __restrict__ first,
                             int shift, JoinBlock blk, bool blocked, const uint64_t* d_n_ref) {
  uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (u >= n_runs) return;
  if (d_n_ref) n_ref = *d_n_ref;
  const uint64_t key = run_keys[u] & key_mask;  // the query run's request does not take part
  uint64_t a = 0, end = n_ref;
  if (first) {
    a = first[key >> shift];
    end = first[(key >> shift) + 1];
  }
  uint64_t b = end;
  while (a < b) {  // lower bound
    uint64_t m = (a + b) >> 1;
    if ((uint64_t)ref_keys[m] < key) a = m + 1;
    else b = m;
  }
  uint64_t lo = a;
  b = end;
  while (a < b) {  // upper bound
    uint64_t m = (a + b) >> 1;
    if ((uint64_t)ref_keys[m] <= key) a = m + 1;
    else b = m;
  }
  uint64_t rc = a - lo;
  uint64_t qc = run_counts[u];
  run_rlo[u] = (uint32_t)lo;
  run_rcount[u] = (uint32_t)rc;
  uint64_t qb = qc;  // entries that expand: the block's share of the run
  if (blocked) {
    const uint32_t q0 = blk.run_qstart[u];
    uint32_t x = q0, y = q0 + (uint32_t)qc;
    while (x < y) {  // first entry at or after the block's first letter
      const uint32_t m = (x + y) >> 1;
      if (blk.q_vals[m] < blk.lo) x = m + 1;
      else y = m;
    }
    const uint32_t b0 = x;
    y = q0 + (uint32_t)qc;
    while (x < y) {  // first entry at or after the block's end
      const uint32_t m = (x + y) >> 1;
      if (blk.q_vals[m] < blk.hi) x = m + 1;
      else y = m;
    }
    blk.run_qlo[u] = b0;
    blk.run_qcount[u] = x - b0;
    qb = x - b0;
  }
  // the cap sees the whole run's count (seed.rs:120-127)
  run_hits[u] = (rc > 0 && qc * rc <= max_expand) ? qb * rc : 0;
}

// One thread per query run: each entry of a run that passes the cap adds
// rcount hits to its target.
__global__ void k_target_hits(const uint32_t* __restrict__ run_counts, const uint32_t* __restrict__ run_qstart,
                              const uint32_t* __restrict__ run_rcount, const uint64_t* __restrict__ run_hits,
                              uint64_t n_runs, const uint32_t* __restrict__ q_vals,
                              const uint32_t* __restrict__ q_owner, unsigned long long* __restrict__ target_hits) {
  const uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (u >= n_runs || run_hits[u] == 0) return;
  const uint32_t q0 = run_qstart[u], qc = run_counts[u], rc = run_rcount[u];
  for (uint32_t e = q0; e < q0 + qc; ++e) atomicAdd(&target_hits[q_owner[q_vals[e]]], (unsigned long long)rc);
}

void launch_target_hits(const uint32_t* run_counts, const uint32_t* run_qstart, const uint32_t* run_rcount,
                        const uint64_t* run_hits, uint64_t n_runs, const uint32_t* q_vals, const uint32_t* q_owner,
                        unsigned long long* target_hits, cudaStream_t st) {
  if (n_runs == 0) return;
  count_launch();
  k_target_hits<<<ceil_div(n_runs, 256), 256, 0, st>>>(run_counts, run_qstart, run_rcount, run_hits, n_runs, q_vals,
                                                        q_owner, target_hits);
  DRG_CUDA(cudaGetLastError());
}

template <typename K>
void join_count(const uint64_t* run_keys, const uint32_t* run_counts, uint64_t n_runs, const K* ref_keys,
                uint64_t n_ref, uint64_t max_expand, uint32_t* run_rlo, uint32_t* run_rcount, uint64_t* run_hits,
                uint64_t key_mask, cudaStream_t st, const uint32_t* first, int shift, const JoinBlock* blk,
                const uint64_t* d_n_ref) {
  if (n_runs == 0) return;
  count_launch();
  k_join_count<K><<<ceil_div(n_runs, 256), 256, 0, st>>>(run_keys, run_counts, n_runs, ref_keys, n_ref, max_expand,
                                                         run_rlo, run_rcount, run_hits, key_mask, first, shift,
                                                         blk ? *blk : JoinBlock{}, blk != nullptr, d_n_ref);
  DRG_CUDA(cudaGetLastError());
}

void launch_join_count(const uint64_t* run_keys, const uint32_t* run_counts, uint64_t n_runs,
                       const uint64_t* ref_keys, uint64_t n_ref, uint64_t max_expand, uint32_t* run_rlo,
                       uint32_t* run_rcount, uint64_t* run_hits, uint64_t key_mask, cudaStream_t st,
                       const uint32_t* first, int shift, const JoinBlock* blk, const uint64_t* d_n_ref) {
  join_count(run_keys, run_counts, n_runs, ref_keys, n_ref, max_expand, run_rlo, run_rcount, run_hits, key_mask, st,
             first, shift, blk, d_n_ref);
}

void launch_join_count(const uint64_t* run_keys, const uint32_t* run_counts, uint64_t n_runs,
                       const uint32_t* ref_keys, uint64_t n_ref, uint64_t max_expand, uint32_t* run_rlo,
                       uint32_t* run_rcount, uint64_t* run_hits, uint64_t key_mask, cudaStream_t st,
                       const uint32_t* first, int shift, const JoinBlock* blk, const uint64_t* d_n_ref) {
  join_count(run_keys, run_counts, n_runs, ref_keys, n_ref, max_expand, run_rlo, run_rcount, run_hits, key_mask, st,
             first, shift, blk, d_n_ref);
}

// coarse[j] = the largest run u < n_runs with run_hit_off[u] <= j << shift,
// for j in [0, nc]: the run of hit h lies in [coarse[h >> shift],
// coarse[(h >> shift) + 1]].
__global__ void k_hit_coarse(const uint64_t* __restrict__ run_hit_off, uint64_t n_runs, int shift, uint64_t nc,
                             uint32_t* __restrict__ coarse) {
  const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (j > nc) return;
  const uint64_t h = j << shift;
  uint64_t lo = 0, hi = n_runs;  // run_hit_off[0] = 0 <= h
  while (hi - lo > 1) {
    const uint64_t m = (lo + hi) >> 1;
    if (run_hit_off[m] <= h) lo = m;
    else hi = m;
  }
  coarse[j] = (uint32_t)lo;
}

void launch_hit_coarse(const uint64_t* run_hit_off, uint64_t n_runs, int shift, uint64_t n_hits, uint32_t* coarse,
                       cudaStream_t st) {
  if (n_runs == 0 || n_hits == 0) return;
  const uint64_t nc = ((n_hits - 1) >> shift) + 1;
  count_launch();
  k_hit_coarse<<<ceil_div((long long)nc + 1, 256), 256, 0, st>>>(run_hit_off, n_runs, shift, nc, coarse);
  DRG_CUDA(cudaGetLastError());
}

__global__ void k_join_expand(JoinExpandArgs a) {
  uint64_t h = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (h >= a.n_hits) return;
  // run u: largest with run_hit_off[u] <= h
  uint64_t lo = 0, hi = a.n_runs;
  if (a.coarse) {
    const uint64_t j = h >> a.coarse_shift;
    lo = a.coarse[j];
    hi = min((uint64_t)a.coarse[j + 1] + 1, a.n_runs);
  }
  while (hi - lo > 1) {
    uint64_t m = (lo + hi) >> 1;
    if (a.run_hit_off[m] <= h) lo = m;
    else hi = m;
  }
  uint64_t u = lo;
  uint64_t k = h - a.run_hit_off[u];
  uint32_t rc = a.run_rcount[u];
  uint64_t qi = a.run_qstart[u] + k / rc;
  uint64_t ri = a.run_rlo[u] + k % rc;
  if (a.hit_keys) {
    uint32_t qg = a.q_vals[qi], rg = a.r_vals[ri];
    uint32_t t = a.q_owner[qg];
    uint32_t s = a.r_owner[rg];
    int64_t qpos = (int64_t)qg - (int64_t)a.q_offsets[t];
    int64_t spos = (int64_t)rg - (int64_t)a.r_offsets[s];
    const HitKeyLayout& L = a.layout;
    uint64_t key = (uint64_t)(t - L.t_base);
    key = (key << L.sb) | (uint64_t)s;
    key = (key << L.db) | (uint64_t)(qpos - spos + L.doff);
    key = (key << L.pb) | (uint64_t)spos;
    a.hit_keys[h] = key;
  } else {
    uint32_t qe = a.q_vals[qi], re = a.r_vals[ri];
    uint32_t* o = a.hits4 + 4 * h;
    o[0] = a.q_seq[qe];
    o[1] = a.q_pos[qe];
    o[2] = a.r_seq[re];
    o[3] = a.r_pos[re];
  }
}

void launch_join_expand(const JoinExpandArgs& a, cudaStream_t st) {
  if (a.n_hits == 0) return;
  count_launch();
  k_join_expand<<<ceil_div(a.n_hits, 256), 256, 0, st>>>(a);
  DRG_CUDA(cudaGetLastError());
}

}  // namespace drg
