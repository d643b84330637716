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

__global__ void k_run_heads(const uint64_t* __restrict__ keys, uint64_t n, int shift, uint8_t* __restrict__ flags) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  flags[i] = (i == 0 || (keys[i] >> shift) != (keys[i - 1] >> shift)) ? 1 : 0;
}

void launch_run_heads(const uint64_t* keys, uint64_t n, int shift, uint8_t* flags, cudaStream_t st) {
  if (n == 0) return;
  count_launch();
  k_run_heads<<<ceil_div(n, 256), 256, 0, st>>>(keys, n, shift, flags);
  DRG_CUDA(cudaGetLastError());
}

// The hits of one (target, subject, diagonal) run, in spos order; returns the
// number of X-drop extensions run.
__device__ __forceinline__ unsigned long long xdrop_run(const XdropArgs& a, uint64_t r, const int8_t* mat) {
  uint64_t i = a.run_head_idx[r];
  const HitKeyLayout L = a.layout;
  const uint64_t run = a.hit_keys[i] >> L.pb;
  const uint32_t t = (uint32_t)(a.hit_keys[i] >> (L.pb + L.db + L.sb));
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

__global__ void k_xdrop_runs(XdropArgs a) {
  __shared__ int8_t mat[625];
  stage_matrix(mat, a.slot);
  const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  unsigned long long nx = 0;
  if (r < a.n_runs) nx = xdrop_run(a, r, mat);
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
  if (p >= a.n_pairs) return;
  const HitKeyLayout L = a.layout;
  uint64_t b = a.pair_head_idx[p], e = a.pair_head_idx[p + 1];
  const uint64_t k0 = a.seg_keys[b];
  const uint32_t t = (uint32_t)(k0 >> (L.pb + L.db + L.sb));
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
