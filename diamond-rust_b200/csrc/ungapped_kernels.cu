// Ungapped X-drop (ungapped.rs:38-88) with the adjacency filter and the
// segment cutoff (search.rs:167-202), and the band merge (search.rs:206-230).
//
// Hits arrive sorted by (target, subject, diagonal, spos) and de-duplicated
// (a repeated hit is skipped by the reference's adjacency rule or yields the
// same rejected segment, so dropping it changes nothing).  One thread owns a
// (target, subject, diagonal) run: the reference's "skip when the last pushed
// segment is on this diagonal and reaches spos" only ever compares hits of
// the same run, so runs are independent.  Kept segments are written at their
// hit's index and compacted afterwards, which preserves the push order.
#include <climits>

#include "kernels.h"

namespace drg {

// One score matrix per context slot (contexts may search concurrently).
__constant__ int8_t c_score[kConstSlots][625];

void upload_score_matrix(const int8_t* s, int slot, cudaStream_t st) {
  DRG_CUDA(cudaMemcpyToSymbolAsync(c_score, s, 625, (size_t)slot * 625, cudaMemcpyHostToDevice, st));
}

// The lanes of a warp look up unrelated residue pairs: from shared memory
// that costs a bank conflict at worst, from constant memory one serialised
// access per distinct address.  Each block stages its slot's matrix first.
__device__ __forceinline__ void stage_matrix(int8_t* mat, int slot) {
  for (int i = threadIdx.x; i < 625; i += blockDim.x) mat[i] = c_score[slot][i];
  __syncthreads();
}
__device__ __forceinline__ int mscore(uint32_t a, uint32_t b, const int8_t* mat) {
  a = a < 24 ? a : 24;
  b = b < 24 ? b : 24;
  return mat[a * 25 + b];
}

__device__ SegmentOut xdrop_dev(const uint8_t* __restrict__ q, uint32_t qlen, const uint8_t* __restrict__ s,
                                uint32_t slen, uint32_t qa, uint32_t sa, int xd, const int8_t* mat) {
  int score = 0, st = 0;
  uint32_t n = 1, delta = 0, len = 0;
  int64_t qi = (int64_t)qa - 1, si = (int64_t)sa - 1;
  while (score - st < xd && qi >= 0 && si >= 0) {
    st += mscore(q[qi], s[si], mat);
    if (st > score) {
      score = st;
      delta = n;
    }
    --qi;
    --si;
    ++n;
  }
  qi = qa;
  si = sa;
  st = score;
  n = 1;
  while (score - st < xd && qi < (int64_t)qlen && si < (int64_t)slen) {
    st += mscore(q[qi], s[si], mat);
    if (st > score) {
      score = st;
      len = n;
    }
    ++qi;
    ++si;
    ++n;
  }
  SegmentOut o;
  o.q_start = qa - delta;
  o.s_start = sa - delta;
  o.len = len + delta;
  o.score = score;
  return o;
}

__global__ void k_run_heads(const uint64_t* __restrict__ keys, uint64_t n, int shift, uint8_t* __restrict__ flags,
                            const int64_t* d_n) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (d_n && i >= (uint64_t)*d_n) {
    flags[i] = 0;
    return;
  }
  flags[i] = (i == 0 || (keys[i] >> shift) != (keys[i - 1] >> shift)) ? 1 : 0;
}

void launch_run_heads(const uint64_t* keys, uint64_t n, int shift, uint8_t* flags, cudaStream_t st,
                      const int64_t* d_n) {
  if (n == 0) return;
  count_launch();
  k_run_heads<<<ceil_div(n, 256), 256, 0, st>>>(keys, n, shift, flags, d_n);
  DRG_CUDA(cudaGetLastError());
}

// The hits of one (target, subject, diagonal) run, in spos order; returns the
// number of X-drop extensions run.
__device__ __forceinline__ unsigned long long xdrop_run(const XdropArgs& a, uint64_t r, const int8_t* mat) {
  uint64_t i = a.run_head_idx[r];
  const HitKeyLayout L = a.layout;
  const uint64_t run = a.hit_keys[i] >> L.pb;
  const uint32_t t = (uint32_t)(a.hit_keys[i] >> (L.pb + L.db + L.sb)) + L.t_base;
  const uint32_t sj = (uint32_t)((a.hit_keys[i] >> (L.pb + L.db)) & ((1ull << L.sb) - 1));
  const int64_t diag = (int64_t)((a.hit_keys[i] >> L.pb) & ((1ull << L.db) - 1)) - L.doff;
  const uint8_t* q = a.q_letters + a.q_offsets[t];
  const uint32_t qlen = (uint32_t)(a.q_offsets[t + 1] - a.q_offsets[t]);
  const uint8_t* s = a.s_letters + a.s_offsets[sj];
  const uint32_t slen = (uint32_t)(a.s_offsets[sj + 1] - a.s_offsets[sj]);
  int64_t last_end = -1;  // s_end of the last kept segment of this run
  unsigned long long nx = 0;  // X-drop extensions run
  for (; i < a.n_hits && (a.hit_keys[i] >> L.pb) == run; ++i) {
    uint32_t spos = (uint32_t)(a.hit_keys[i] & ((1ull << L.pb) - 1));
    a.keep[i] = 0;
    if (last_end >= (int64_t)spos) continue;
    uint32_t qpos = (uint32_t)(diag + spos);
    SegmentOut seg = xdrop_dev(q, qlen, s, slen, qpos, spos, a.xdrop, mat);
    ++nx;
    if (seg.score >= a.cutoff) {
      a.seg[i] = seg;
      a.keep[i] = 1;
      last_end = (int64_t)seg.s_start + seg.len;
    }
  }
  return nx;
}

// One direction of an X-drop extension in flight (ungapped.rs:46-83): steps
// taken so far, the running score, the best score and the step that reached
// it first.  Left: step k compares (qa-1-k, sa-1-k); right: (qa+k, sa+k).
struct XdropDir {
  const uint8_t* q;
  const uint8_t* s;
  int64_t qa, sa;
  uint32_t bound;  // steps before a sequence end
  uint32_t k;      // steps taken
  int st, score;
  uint32_t best;   // steps when the best was first reached (delta / len)
  bool left;
};

// An extension still running after this many cells in one direction is
// finished by the whole warp.  Random hits mostly stop within 20-60 cells:
// with a limit of 32 many of them took the warp path (X-drop stage 0.57 ->
// 0.73 ms at 1,000 queries); true homologies run for hundreds.
constexpr uint32_t kXdropSerialSteps = 128;

// Serial steps, at most `limit`; true when the direction has stopped (the
// reference's loop condition failed or a sequence ended).
__device__ __forceinline__ bool xdrop_steps(XdropDir& d, int xd, uint32_t limit, const int8_t* mat) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (!(d.score - d.st < xd && d.k < d.bound)) return true;
    const int64_t qi = d.left ? d.qa - 1 - d.k : d.qa + d.k, si = d.left ? d.sa - 1 - d.k : d.sa + d.k;
    d.st += mscore(d.q[qi], d.s[si], mat);
    ++d.k;
    if (d.st > d.score) {
      d.score = d.st;
      d.best = d.k;
    }
  }
  return !(d.score - d.st < xd && d.k < d.bound);
}

// The whole warp runs one lane's direction to its end, 32 steps at a time:
// lane l scores step k0 + l; prefix sums give the running score after each
// step, prefix maxima the best before it; the first step whose condition
// fails (or that is past a sequence end) ends the direction; the best's
// first occurrence among the steps taken is where the reference's strict
// "st > score" last fired.  Every lane returns the same state.
__device__ XdropDir xdrop_warp(XdropDir d, int xd, const int8_t* mat) {
  const uint32_t lane = threadIdx.x & 31;
  for (;;) {
    const uint32_t k = d.k + lane;
    const bool valid = k < d.bound;
    int sc = 0;
    if (valid) {
      const int64_t qi = d.left ? d.qa - 1 - k : d.qa + k, si = d.left ? d.sa - 1 - k : d.sa + k;
      sc = mscore(d.q[qi], d.s[si], mat);
    }
    int sum = sc;  // inclusive prefix sum of the step scores
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xFFFFFFFFu, sum, o);
      if (lane >= (uint32_t)o) sum += y;
    }
    const int st_after = d.st + sum;  // running score after this lane's step
    int mx = valid ? st_after : INT_MIN;  // inclusive prefix max of the running score
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xFFFFFFFFu, mx, o);
      if (lane >= (uint32_t)o) mx = max(mx, y);
    }
    const int mx_prev = __shfl_up_sync(0xFFFFFFFFu, mx, 1);  // every lane takes part in the shuffle
    const int best_before = max(d.score, lane == 0 ? INT_MIN : mx_prev);
    const int st_before = st_after - sc;
    const uint32_t stop = __ballot_sync(0xFFFFFFFFu, !valid || !(best_before - st_before < xd));
    const uint32_t taken = stop ? (uint32_t)(__ffs(stop) - 1) : 32u;
    if (taken > 0) {
      const int new_st = __shfl_sync(0xFFFFFFFFu, st_after, taken - 1);
      const int top = max(d.score, __shfl_sync(0xFFFFFFFFu, mx, taken - 1));
      if (top > d.score) {
        const uint32_t first = __ballot_sync(0xFFFFFFFFu, lane < taken && st_after == top);
        d.best = d.k + (uint32_t)__ffs(first);  // steps up to and including the first maximum
        d.score = top;
      }
      d.st = new_st;
      d.k += taken;
    }
    if (taken < 32) return d;
  }
}

// One thread per (target, subject, diagonal) run, as xdrop_run, except that
// an extension still going after kXdropSerialSteps cells in one direction is
// finished by the whole warp (xdrop_warp), so that a long true-homology
// extension does not hold 31 idle lanes.  The hits of a run, the skip rule
// (search.rs:184-191) and the cutoff stay in order per lane.
__global__ void k_xdrop_runs(XdropArgs a) {
  __shared__ int8_t mat[625];
  stage_matrix(mat, a.slot);
  const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  const HitKeyLayout L = a.layout;
  if (a.d_n_hits) a.n_hits = (uint64_t)*a.d_n_hits;
  if (a.d_n_runs) a.n_runs = (uint64_t)*a.d_n_runs;
  bool live = r < a.n_runs;  // the lane still has hits to extend
  uint64_t i = 0, run = 0;
  const uint8_t *q = nullptr, *s = nullptr;
  uint32_t qlen = 0, slen = 0;
  int64_t diag = 0, last_end = -1;
  if (live) {
    i = a.run_head_idx[r];
    run = a.hit_keys[i] >> L.pb;
    const uint32_t t = (uint32_t)(a.hit_keys[i] >> (L.pb + L.db + L.sb)) + L.t_base;
    const uint32_t sj = (uint32_t)((a.hit_keys[i] >> (L.pb + L.db)) & ((1ull << L.sb) - 1));
    diag = (int64_t)((a.hit_keys[i] >> L.pb) & ((1ull << L.db) - 1)) - L.doff;
    q = a.q_letters + a.q_offsets[t];
    qlen = (uint32_t)(a.q_offsets[t + 1] - a.q_offsets[t]);
    s = a.s_letters + a.s_offsets[sj];
    slen = (uint32_t)(a.s_offsets[sj + 1] - a.s_offsets[sj]);
  }
  bool ext = false;     // an extension is in flight
  XdropDir d{};         // its current direction
  int left_score = 0;   // the left direction's best (the right one starts there)
  uint32_t delta = 0;   // the left direction's best step
  uint32_t qpos = 0, spos = 0;
  unsigned long long nx = 0;
  for (;;) {
    bool needs_warp = false;
    while (live) {
      if (!ext) {
        // the next hit of the run that the skip rule lets through
        while (i < a.n_hits && (a.hit_keys[i] >> L.pb) == run) {
          spos = (uint32_t)(a.hit_keys[i] & ((1ull << L.pb) - 1));
          a.keep[i] = 0;
          if (last_end < (int64_t)spos) break;
          ++i;
        }
        if (!(i < a.n_hits && (a.hit_keys[i] >> L.pb) == run)) {
          live = false;
          break;
        }
        qpos = (uint32_t)(diag + spos);
        d = XdropDir{q, s, qpos, spos, min(qpos, spos), 0, 0, 0, 0, true};
        ext = true;
        ++nx;
      }
      if (!xdrop_steps(d, a.xdrop, kXdropSerialSteps, mat)) {
        needs_warp = true;
        break;
      }
      if (d.left) {  // the right direction starts from the left's best
        left_score = d.score;
        delta = d.best;
        d = XdropDir{q, s, qpos, spos, min(qlen - qpos, slen - spos), 0, left_score, left_score, 0, false};
      } else {
        SegmentOut seg;
        seg.q_start = qpos - delta;
        seg.s_start = spos - delta;
        seg.len = d.best + delta;
        seg.score = d.score;
        if (seg.score >= a.cutoff) {
          a.seg[i] = seg;
          a.keep[i] = 1;
          last_end = (int64_t)seg.s_start + seg.len;
        }
        ++i;
        ext = false;
      }
    }
    const uint32_t help = __ballot_sync(0xFFFFFFFFu, needs_warp);
    if (__ballot_sync(0xFFFFFFFFu, live) == 0) break;
    // the long directions, one at a time, by the whole warp
    for (uint32_t m = help; m; m &= m - 1) {
      const int src = __ffs(m) - 1;
      XdropDir w;
      w.q = reinterpret_cast<const uint8_t*>(__shfl_sync(0xFFFFFFFFu, reinterpret_cast<uint64_t>(d.q), src));
      w.s = reinterpret_cast<const uint8_t*>(__shfl_sync(0xFFFFFFFFu, reinterpret_cast<uint64_t>(d.s), src));
      w.qa = __shfl_sync(0xFFFFFFFFu, d.qa, src);
      w.sa = __shfl_sync(0xFFFFFFFFu, d.sa, src);
      w.bound = __shfl_sync(0xFFFFFFFFu, d.bound, src);
      w.k = __shfl_sync(0xFFFFFFFFu, d.k, src);
      w.st = __shfl_sync(0xFFFFFFFFu, d.st, src);
      w.score = __shfl_sync(0xFFFFFFFFu, d.score, src);
      w.best = __shfl_sync(0xFFFFFFFFu, d.best, src);
      w.left = __shfl_sync(0xFFFFFFFFu, (int)d.left, src) != 0;
      w = xdrop_warp(w, a.xdrop, mat);
      if ((int)lane == src) d = w;  // the direction has stopped: the lane's loop moves on
    }
  }
  warp_sum_atomic(a.xdrop_count, nx);
}

void launch_xdrop_runs(const XdropArgs& a, cudaStream_t st) {
  if (a.n_runs == 0) return;
  count_launch();
  k_xdrop_runs<<<ceil_div(a.n_runs, 128), 128, 0, st>>>(a);
  DRG_CUDA(cudaGetLastError());
}

__global__ void k_xdrop_jobs(const drg_xdrop_job* __restrict__ jobs, uint64_t n, const uint8_t* __restrict__ ql,
                             const uint64_t* __restrict__ qo, const uint8_t* __restrict__ sl,
                             const uint64_t* __restrict__ so, int xd, drg_segment* __restrict__ out, int slot) {
  __shared__ int8_t mat[625];
  stage_matrix(mat, slot);
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  drg_xdrop_job j = jobs[i];
  SegmentOut g = xdrop_dev(ql + qo[j.query], (uint32_t)(qo[j.query + 1] - qo[j.query]), sl + so[j.subject],
                           (uint32_t)(so[j.subject + 1] - so[j.subject]), (uint32_t)j.qa, (uint32_t)j.sa, xd, mat);
  drg_segment r;
  r.q_start = g.q_start;
  r.s_start = g.s_start;
  r.len = g.len;
  r.score = g.score;
  r.pad = 0;
  out[i] = r;
}

void launch_xdrop_jobs(const drg_xdrop_job* jobs, uint64_t n, const uint8_t* ql, const uint64_t* qo,
                       const uint8_t* sl, const uint64_t* so, int xd, drg_segment* out, int slot, cudaStream_t st) {
  if (n == 0) return;
  count_launch();
  k_xdrop_jobs<<<ceil_div(n, 128), 128, 0, st>>>(jobs, n, ql, qo, sl, so, xd, out, slot);
  DRG_CUDA(cudaGetLastError());
}

// Band order of one pair, search.rs:206-230, for segments given in push order
// (diagonal ascending, spos ascending):
//  - bands are maximal runs of segments whose [diag - band, diag + band]
//    intervals chain-overlap in diagonal order;
//  - a band's best segment is the first, in that order, with the top score
//    (the reference's stable sorts visit equal diagonals in push order);
//  - bands are ordered by best score, descending, ties by diagonal (the
//    reference's insertion sort is stable for the <= 20 bands a pair has;
//    longer lists with ties follow the same rule here).
// The window of gapped_hsp (search.rs:303-312) is applied to each band.
__global__ void k_build_bands(BandArgs a) {
  uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (p >= a.n_pairs || (a.d_n_pairs && p >= (uint64_t)*a.d_n_pairs)) return;
  const HitKeyLayout L = a.layout;
  uint64_t b = a.pair_head_idx[p], e = a.pair_head_idx[p + 1];
  const uint64_t k0 = a.seg_keys[b];
  const uint32_t t = (uint32_t)(k0 >> (L.pb + L.db + L.sb)) + L.t_base;
  const uint32_t sj = (uint32_t)((k0 >> (L.pb + L.db)) & ((1ull << L.sb) - 1));
  const uint32_t qlen = (uint32_t)(a.q_offsets[t + 1] - a.q_offsets[t]);
  // band_for (gapped.rs:27-32)
  const uint32_t th[7] = {50, 100, 150, 200, 250, 350, 500};
  const int bw[8] = {12, 16, 30, 30, 30, 40, 64, 64};
  int bucket = 0;
  for (int k = 0; k < 7; ++k) bucket += qlen >= th[k];
  const int band = bw[bucket];
  // pass 1: merge in diagonal order; bands written at [b, b + nb)
  uint64_t nb = 0;
  int64_t cur_d0 = 0, cur_d1 = 0;
  int32_t cur_best = 0;
  uint32_t cur_aq = 0;
  for (uint64_t i = b; i < e; ++i) {
    int64_t diag = (int64_t)((a.seg_keys[i] >> L.pb) & ((1ull << L.db) - 1)) - L.doff;
    int32_t sc = a.segs[i].score;
    int64_t b0 = diag - band, b1 = diag + band;
    if (nb > 0 && b0 <= cur_d1) {
      if (b1 > cur_d1) cur_d1 = b1;
      if (sc > cur_best) {
        cur_best = sc;
        cur_aq = a.segs[i].q_start;
      }
    } else {
      if (nb > 0) {
        Band& o = a.bands[b + nb - 1];
        o.d0 = (int32_t)cur_d0;
        o.d1 = (int32_t)cur_d1;
        o.best_score = cur_best;
        o.q0 = cur_aq;  // anchor query position until the window is set
      }
      ++nb;
      cur_d0 = b0;
      cur_d1 = b1;
      cur_best = sc;
      cur_aq = a.segs[i].q_start;
    }
  }
  {
    Band& o = a.bands[b + nb - 1];
    o.d0 = (int32_t)cur_d0;
    o.d1 = (int32_t)cur_d1;
    o.best_score = cur_best;
    o.q0 = cur_aq;
  }
  // pass 2: stable insertion sort by best score, descending
  for (uint64_t i = b + 1; i < b + nb; ++i) {
    Band x = a.bands[i];
    uint64_t j = i;
    while (j > b && a.bands[j - 1].best_score < x.best_score) {
      a.bands[j] = a.bands[j - 1];
      --j;
    }
    a.bands[j] = x;
  }
  // pass 3: windows (gapped_hsp), identity fields
  for (uint64_t i = b; i < b + nb; ++i) {
    Band& o = a.bands[i];
    uint64_t row_cells = (uint64_t)(o.d1 - o.d0) + 1;
    uint64_t max_rows = 16000000ull / row_cells;
    if (max_rows < 2ull * band + 16) max_rows = 2ull * band + 16;
    uint64_t anchor_q = o.q0;
    uint64_t q0 = 0, q1 = qlen;
    if (q1 - q0 > max_rows) {
      q0 = anchor_q >= max_rows / 2 ? anchor_q - max_rows / 2 : 0;
      q1 = q0 + max_rows < qlen ? q0 + max_rows : qlen;
      q0 = q1 >= max_rows ? q1 - max_rows : 0;
    }
    o.target = t;
    o.subject = sj;
    o.q0 = (uint32_t)q0;
    o.n = (uint32_t)(q1 - q0);
    o.d0 -= (int32_t)q0;
    o.d1 -= (int32_t)q0;
    o.rank = (uint32_t)(i - b);
    o.pair = (uint32_t)p;
    o.pad = 0;
    a.valid[i] = 1;
  }
  for (uint64_t i = b + nb; i < e; ++i) a.valid[i] = 0;
}

void launch_build_bands(const BandArgs& a, cudaStream_t st) {
  if (a.n_pairs == 0) return;
  count_launch();
  k_build_bands<<<ceil_div(a.n_pairs, 128), 128, 0, st>>>(a);
  DRG_CUDA(cudaGetLastError());
}

}  // namespace drg
