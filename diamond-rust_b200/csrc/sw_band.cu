// Banded affine Smith-Waterman (gapped.rs:67-280) with lanes of a warp on
// one band: the wide bands of the score pass and the traceback pass of the
// HSPs that survive the E-value gate, whose few, long bands leave an
// inter-band warp nearly empty.  Two mappings: the block kernel (k_sw_band,
// below) and rotating strips (k_sw_rot, further down), which the launcher
// picks by width.
//
// Block kernel (intra-band, systolic): lane l runs strip 32b + l of the band (16
// DP rows, the same s16x2 pair layout and column recurrence as the packed
// inter-band kernel) in block b of 32 strips.  Strip k + 1 at relative column
// c needs the (H, E) of strip k's last row at strip k's relative column c + 16,
// which strip k produces at its step c + 17.  So lane l runs its step c at
// warp time T = c + 18 l and takes that word from lane l - 1's output of time
// T - 1 with one shuffle; the D operand is the word of the step before.  Lane
// 0 of block b + 1 reads lane 31's words of block b from shared memory.  At
// any time only one lane is in its first 16 steps and one in its last 16, but
// as lanes are at different columns the band-edge masks are computed per
// lane at run time.
//
// Results (trace nibbles, score, first row-major maximum) equal the packed
// inter-band kernel's and hence the reference's; in trace mode each band is
// walked (sw_walk.cuh) right after its DP, through nibbles laid out with a
// unit stride between column steps.
#include "kernels.h"
#include "sw_common.cuh"
#include "sw_walk.cuh"

namespace drg {

namespace {

using namespace sw;

constexpr int kLag = kRows + 2;   // steps between consecutive lanes
constexpr int kLaneProf = 424;    // 26 residues x 16 rows, padded: per-lane strip profile
constexpr int kBandWarps = 4;

// Half masks of pair p at relative column c: sign of (c - p, c - p - 9)
// replicated over each half, i.e. 0xFFFF where the row's cell is left of
// column 0 of its band (left) or, given cw = c - W, still inside it (right).
__device__ __forceinline__ uint32_t neg_mask(uint32_t v) { return prmt(v, 0u, 0xBB99u); }

// One column step of a strip at run-time column c (band width W); rw is the
// (H, E) word of the row above at column c.  Returns the (H, E) word of row 15
// at column c - 1.
template <bool TR>
__device__ __forceinline__ uint32_t band_step(Regs<TR>& R, const Lane& L, int c, uint32_t cc2, uint32_t cw2,
                                              const uint8_t* __restrict__ prof, uint32_t rw, uint32_t noc2,
                                              uint32_t nge2, uint2* __restrict__ trace) {
  const uint32_t res = subject_residue(L, L.jbase + c - 1);
  const uint2 lo8 = *reinterpret_cast<const uint2*>(prof + res * kRows);
  const uint2 hi8 = *reinterpret_cast<const uint2*>(prof + R.res_prev * kRows + 8);
  R.res_prev = res;
  const uint32_t htop = prmt(rw, R.H[kPairs - 1], 0x5410);
  uint32_t e_up = prmt(rw, R.E7, 0x5432);
  uint32_t hm_up = add2(htop, noc2);
  uint32_t hd = R.htop_old;
  uint32_t tr_lo = 0, tr_hi = 0;
  const uint32_t colpair = TR ? ((uint32_t)c | ((uint32_t)(c - 1) << 16)) : 0u;
#pragma unroll
  for (int p = 0; p < kPairs; ++p) {
    const uint32_t sc = prmt(p < 4 ? lo8.x : lo8.y, p < 4 ? hi8.x : hi8.y, pick_sel(p & 3));
    const uint32_t d = add2(hd, sc);
    uint32_t e, f, h;
    if (!TR) {
      e = __viaddmax_s16x2(e_up, nge2, hm_up);
      f = __viaddmax_s16x2(R.F[p], nge2, R.Hm[p]);
      h = __vimax3_s16x2_relu(d, e, f);
    } else {
      const uint32_t te = add2(e_up, nge2);
      const uint32_t tf = add2(R.F[p], nge2);
      e = max2(te, hm_up);
      f = max2(tf, R.Hm[p]);
      const uint32_t m1 = max2_relu(d, 0u);
      const uint32_t ce = __vcmpgts2(e, m1);
      const uint32_t m2 = max2(e, m1);
      const uint32_t cf = __vcmpgts2(f, m2);
      h = max2(f, m2);
      const uint32_t cd = __vcmpgts2(d, 0u);
      const uint32_t ee = __vcmpgts2(te, hm_up);
      const uint32_t fe = __vcmpgts2(tf, R.Hm[p]);
      uint32_t bits = ((cf | (cd & ~ce)) & 0x00010001u) | ((cf | ce) & 0x00020002u) | (ee & 0x00040004u) |
                      (fe & 0x00080008u);
      const uint32_t byte = (bits & 0xFu) | ((bits >> 12) & 0xF0u);
      if (p < 4) tr_lo |= byte << (8 * (p & 3));
      else tr_hi |= byte << (8 * (p & 3));
    }
    // thresholds (p, p + 9) per half, as s16x2
    const uint32_t thr = (uint32_t)(uint16_t)(-p) | ((uint32_t)(uint16_t)(-(p + 9)) << 16);
    const uint32_t left = neg_mask(add2(cc2, thr));    // left of the band: no score, F = -inf
    const uint32_t inside = neg_mask(add2(cw2, thr));  // not right of the band; else no score, E = -inf
    h = h & ~left & inside;
    f = sel2(f, ~left, kNeg2);
    e = sel2(e, inside, kNeg2);
    const uint32_t hm = add2(h, noc2);
    if (!TR) {
      R.rowmax[p] = max2(R.rowmax[p], h);
    } else {
      const uint32_t gt = __vcmpgts2(h, R.rowmax[p]);
      R.rowmax[p] = max2(R.rowmax[p], h);
      R.rowcol[p] = (R.rowcol[p] & ~gt) | (colpair & gt);
    }
    hd = R.H[p];
    R.H[p] = h;
    R.Hm[p] = hm;
    R.F[p] = f;
    hm_up = hm;
    e_up = e;
  }
  R.E7 = e_up;
  R.htop_old = htop;
  if (TR) *trace = make_uint2(tr_lo, tr_hi);
  return prmt(R.H[kPairs - 1], R.E7, 0x7632);
}

template <bool TR>
__global__ void __launch_bounds__(kBandWarps * 32) k_sw_band(SwBandArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int8_t* mat = reinterpret_cast<int8_t*>(smem);
  for (int i = threadIdx.x; i < 625; i += blockDim.x) mat[i] = a.scores625[i];
  __syncthreads();
  const uint64_t t = a.lo + (uint64_t)blockIdx.x * kBandWarps + warp;
  if (t >= a.hi) return;  // warp-uniform
  uint8_t* prof = smem + 640 + (warp * 32 + lane) * kLaneProf;
  uint32_t* xbuf = reinterpret_cast<uint32_t*>(smem + 640 + kBandWarps * 32 * kLaneProf) +
                   (size_t)warp * 2 * a.xbuf_words;
  const SwBandJob job = a.jobs[t];
  const Band band = a.bands[job.band];
  const int W = band.d1 - band.d0 + 1;
  const int steps = W + kRows;  // column steps of one strip
  const uint8_t* q = a.q_letters + a.q_offsets[band.target] + band.q0;
  const int n = (int)band.n;
  Lane L;
  L.s = a.s_letters + a.s_offsets[band.subject];
  L.m = (int)(a.s_offsets[band.subject + 1] - a.s_offsets[band.subject]);
  const uint32_t noc2 = (uint32_t)(uint16_t)(-(a.gap_open + a.gap_extend)) * 0x10001u;
  const uint32_t nge2 = (uint32_t)(uint16_t)(-a.gap_extend) * 0x10001u;
  int best = 0, best_i = 0, best_j = 0;
  const int n_strips = (int)job.n_strips;
  for (int b0 = 0, blk = 0; b0 < n_strips; b0 += 32, ++blk) {
    const int cnt = min(32, n_strips - b0);
    const bool has = lane < cnt;
    const bool feeds_next = b0 + 32 < n_strips;
    const int i0 = (int)job.row_first + kRows * (b0 + lane);
    // this lane's strip profile: prof[res * 16 + r] = S(q[i0 + r - 1], res)
    if (has) {
      uint32_t qr[kRows];
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int i = i0 + r;
        qr[r] = i > n ? 255u : (uint32_t)min((uint32_t)q[i - 1], 24u);
      }
      for (int res = 0; res < 26; ++res) {
#pragma unroll
        for (int r4 = 0; r4 < 4; ++r4) {
          uint32_t w = 0;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const uint32_t r = qr[r4 * 4 + k];
            const int v = (res == 25 || r == 255u) ? kSentinelScore : mat[r * 25 + res];
            w |= ((uint32_t)(uint8_t)(int8_t)v) << (8 * k);
          }
          *reinterpret_cast<uint32_t*>(prof + res * kRows + r4 * 4) = w;
        }
      }
    }
    __syncwarp();
    const uint32_t* xin = xbuf + (size_t)((blk + 1) & 1) * a.xbuf_words;  // lane 31's words of the last block
    uint32_t* xout = xbuf + (size_t)(blk & 1) * a.xbuf_words;
    L.jbase = i0 - band.d1;
    Regs<TR> R;
    uint2* tr = TR ? a.trace + job.trace_off + (uint64_t)(b0 + lane) * steps : nullptr;
    // the word of the row above at column -1 (only lane 0 uses its own)
    uint32_t rw_prev = blk == 0 ? 0xC0000000u : xin[kRows];
    uint32_t out_prev = kNeg2;
    const int t_end = steps + kLag * (cnt - 1);
    for (int T = 0; T < t_end; ++T) {
      const int c = T - kLag * lane;
      uint32_t rw = __shfl_up_sync(0xFFFFFFFFu, out_prev, 1);
      if (lane == 0) {
        if (blk == 0) rw = c < W - 1 ? 0xC0000000u : kNeg2;  // row 0 of the reference: H = 0, E = -inf
        else rw = c + kRows + 1 < steps ? xin[c + kRows + 1] : kNeg2;
      }
      uint32_t out = kNeg2;  // a finished strip passes -inf to the next
      if (has && (unsigned)c < (unsigned)steps) {
        if (c == 0) {
#pragma unroll
          for (int p = 0; p < kPairs; ++p) {
            R.H[p] = 0;
            R.Hm[p] = kNeg2;
            R.F[p] = kNeg2;
            R.rowmax[p] = 0;
            if (TR) R.rowcol[p] = 0;
          }
          R.E7 = kNeg2;
          R.htop_old = rw_prev & 0xFFFFu;
          const int jm1 = L.jbase - 2;
          R.res_prev = subject_residue(L, jm1);
        }
        const uint32_t cc2 = (uint32_t)c * 0x10001u;
        const uint32_t cw2 = (uint32_t)(uint16_t)(c - W) * 0x10001u;
        out = band_step<TR>(R, L, c, cc2, cw2, prof, rw, noc2, nge2, TR ? tr + c : nullptr);
        if (feeds_next && lane == 31) xout[c] = out;
        if (c == steps - 1) {
#pragma unroll
          for (int r = 0; r < kRows; ++r) {
            const int v = r < kPairs ? lo16(R.rowmax[r]) : hi16(R.rowmax[r - kPairs]);
            if (v > best) {
              best = v;
              best_i = i0 + r;
              if (TR) best_j = L.jbase + (r < kPairs ? lo16(R.rowcol[r]) : hi16(R.rowcol[r - kPairs]));
            }
          }
        }
      }
      rw_prev = rw;
      out_prev = out;
    }
    __syncwarp();
  }
  // first row-major maximum over the lanes: highest score, then lowest row
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int ob = __shfl_xor_sync(0xFFFFFFFFu, best, o);
    const int oi = __shfl_xor_sync(0xFFFFFFFFu, best_i, o);
    const int oj = __shfl_xor_sync(0xFFFFFFFFu, best_j, o);
    if (ob > best || (ob == best && ob > 0 && oi < best_i)) {
      best = ob;
      best_i = oi;
      best_j = oj;
    }
  }
  if (best == 0) best_i = best_j = 0;
  if (lane != 0) return;
  if (!TR) {
    a.score[job.band] = best;
    if (a.best_row) a.best_row[job.band] = best_i;
  } else {
    TraceBand tb;
    tb.trace_off = job.trace_off;
    tb.row_first = job.row_first;
    tb.width = (uint32_t)W;
    tb.score = best;
    tb.best_i = best_i;
    tb.best_j = best_j;
    tb.stride = 1;  // consecutive column steps
    a.tband[job.band] = tb;
    // the walk, while the SM's other warps run DP; the warp's exchange
    // buffer (free now) holds its 8-word trace window
    walk_band(a.walk, job.band, band, tb, mat, reinterpret_cast<uint2*>(xbuf), 1);
  }
}

// ---- rotating strips: G lanes per band, several bands per warp --------------
//
// One band needs about (W + 16) / 18 lanes at a time: strip s + 1 can start 18
// steps after strip s (the lag above) and a strip lasts W + 16 steps.  So a
// warp holds 32 / G bands, G lanes each, and lane l of a group runs strips l,
// l + G, l + 2G, ...: strip s starts at group time Lag * s on lane s mod G,
// and takes the row above from lane (s - 1) mod G by a shuffle.  Lag is 18
// (or 19 for 8-lane groups of widths 128-134) under two conditions on the
// width: a lane's strips do not overlap (W + 16 <= G * Lag), and a strip
// has passed its last column (and sends -inf) before its lane starts the
// next strip while its successor still reads it (W - 1 <= (G - 1) * Lag).
// Routes: G = 8 for W <= 134, 16 for W <= 271, 32 for W <= 559; wider bands
// use the block kernel above.
constexpr int kRotWarps = 4;

template <int G>
__device__ __forceinline__ int rot_lag(int w_max) {
  return (G == 8 && w_max > 127) ? kLag + 1 : kLag;
}

template <int G, bool TR>
__global__ void __launch_bounds__(kRotWarps * 32) k_sw_rot(SwBandArgs a) {
  constexpr int NG = 32 / G;  // bands per warp
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = lane / G, gl = lane % G;
  int8_t* mat = reinterpret_cast<int8_t*>(smem);
  for (int i = threadIdx.x; i < 625; i += blockDim.x) mat[i] = a.scores625[i];
  __syncthreads();
  uint8_t* prof_base = smem + 640 + (size_t)(warp * 32) * kLaneProf;  // lane x's profile at x * kLaneProf
  uint8_t* prof = prof_base + (size_t)lane * kLaneProf;
  uint2* win = reinterpret_cast<uint2*>(smem + 640 + (size_t)kRotWarps * 32 * kLaneProf) +
               (size_t)(warp * NG + grp) * kWalkWindow;  // the group's walk window
  const uint64_t t = a.lo + ((uint64_t)blockIdx.x * kRotWarps + warp) * NG + grp;
  const bool has_job = t < a.hi;
  SwBandJob job{};
  Band band{};
  if (has_job) {
    job = a.jobs[t];
    band = a.bands[job.band];
  }
  const int W = has_job ? band.d1 - band.d0 + 1 : 0;
  const int steps = W + kRows;
  const int S = has_job ? (int)job.n_strips : 0;
  const int lag = rot_lag<G>(__reduce_max_sync(0xFFFFFFFFu, W));
  const int t_group = S > 0 ? lag * (S - 1) + steps : 0;
  const int t_end = __reduce_max_sync(0xFFFFFFFFu, t_group);
  const uint8_t* q = has_job ? a.q_letters + a.q_offsets[band.target] + band.q0 : a.q_letters;
  const int n = has_job ? (int)band.n : 0;
  Lane L;
  L.s = has_job ? a.s_letters + a.s_offsets[band.subject] : a.s_letters;
  L.m = has_job ? (int)(a.s_offsets[band.subject + 1] - a.s_offsets[band.subject]) : 0;
  const uint32_t noc2 = (uint32_t)(uint16_t)(-(a.gap_open + a.gap_extend)) * 0x10001u;
  const uint32_t nge2 = (uint32_t)(uint16_t)(-a.gap_extend) * 0x10001u;
  const int src = grp * G + (gl + G - 1) % G;  // the lane of the previous strip
  int best = 0, best_i = 0, best_j = 0;
  Regs<TR> R;
  int s = gl;            // this lane's current (or next) strip
  int c = -lag * gl;     // its column: strip s starts at group time lag * s
  int i0 = 0;
  uint2* tr = nullptr;
  uint32_t rw_prev = 0xC0000000u, out_prev = kNeg2, out_prev2 = kNeg2;
  int ph = 0, s0 = 0;  // group time modulo lag; the strip starting at the next multiple
  // the query letters of strip s0's rows, loaded one strip ahead of the
  // profile they feed (the loads' latency then hides behind lag steps)
  uint32_t qr[kRows];
  auto load_rows = [&](int sk) {
    const int ib = (int)job.row_first + kRows * sk;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int i = ib + r;
      qr[r] = (sk >= S || i > n) ? 255u : (uint32_t)min((uint32_t)q[i - 1], 24u);
    }
  };
  load_rows(0);
  for (int T = 0; T < t_end; ++T) {
    // The strip starting now (group time lag * s0) gets its profile from the
    // whole group: lane x of the group fills residues x, x + G, ...
    if (ph == 0) {
      if (s0 < S) {
        uint8_t* dst = prof_base + (size_t)(grp * G + s0 % G) * kLaneProf;
        for (int res = gl; res < 26; res += G) {
#pragma unroll
          for (int r4 = 0; r4 < 4; ++r4) {
            uint32_t w = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const uint32_t r = qr[r4 * 4 + k];
              const int v = (res == 25 || r == 255u) ? kSentinelScore : mat[r * 25 + res];
              w |= ((uint32_t)(uint8_t)(int8_t)v) << (8 * k);
            }
            *reinterpret_cast<uint32_t*>(dst + res * kRows + r4 * 4) = w;
          }
        }
      }
      ++s0;
      load_rows(s0);
      __syncwarp();
    }
    if (++ph == lag) ph = 0;
    // the row above at this lane's column: the previous strip's word, or
    // row 0 of the reference for the band's first strip
    uint32_t rw = __shfl_sync(0xFFFFFFFFu, lag == kLag ? out_prev : out_prev2, src);
    if (s == 0) rw = c < W - 1 ? 0xC0000000u : kNeg2;
    uint32_t out = kNeg2;  // a lane between strips passes -inf
    if (s < S && c >= 0 && c < steps) {
      if (c == 0) {
        i0 = (int)job.row_first + kRows * s;
        L.jbase = i0 - band.d1;
        if (TR) tr = a.trace + job.trace_off + (uint64_t)s * steps;
#pragma unroll
        for (int p = 0; p < kPairs; ++p) {
          R.H[p] = 0;
          R.Hm[p] = kNeg2;
          R.F[p] = kNeg2;
          R.rowmax[p] = 0;
          if (TR) R.rowcol[p] = 0;
        }
        R.E7 = kNeg2;
        R.htop_old = s == 0 ? 0u : (rw_prev & 0xFFFFu);
        R.res_prev = subject_residue(L, L.jbase - 2);
      }
      const uint32_t cc2 = (uint32_t)c * 0x10001u;
      const uint32_t cw2 = (uint32_t)(uint16_t)(c - W) * 0x10001u;
      out = band_step<TR>(R, L, c, cc2, cw2, prof, rw, noc2, nge2, TR ? tr + c : nullptr);
      if (c == steps - 1) {
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
          const int v = r < kPairs ? lo16(R.rowmax[r]) : hi16(R.rowmax[r - kPairs]);
          if (v > best) {
            best = v;
            best_i = i0 + r;
            if (TR) best_j = L.jbase + (r < kPairs ? lo16(R.rowcol[r]) : hi16(R.rowcol[r - kPairs]));
          }
        }
      }
    }
    rw_prev = rw;
    out_prev2 = out_prev;
    out_prev = out;
    if (++c == G * lag) {  // this lane's next strip
      c = 0;
      s += G;
    }
  }
  __syncwarp();
  // first row-major maximum over the group: highest score, then lowest row
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    const int ob = __shfl_xor_sync(0xFFFFFFFFu, best, o);
    const int oi = __shfl_xor_sync(0xFFFFFFFFu, best_i, o);
    const int oj = __shfl_xor_sync(0xFFFFFFFFu, best_j, o);
    if (ob > best || (ob == best && ob > 0 && oi < best_i)) {
      best = ob;
      best_i = oi;
      best_j = oj;
    }
  }
  if (best == 0) best_i = best_j = 0;
  if (gl != 0 || !has_job) return;
  if (!TR) {
    a.score[job.band] = best;
    if (a.best_row) a.best_row[job.band] = best_i;
  } else {
    TraceBand tb;
    tb.trace_off = job.trace_off;
    tb.row_first = job.row_first;
    tb.width = (uint32_t)W;
    tb.score = best;
    tb.best_i = best_i;
    tb.best_j = best_j;
    tb.stride = 1;
    a.tband[job.band] = tb;
    walk_band(a.walk, job.band, band, tb, mat, win, 1);
  }
}

}  // namespace

template <int G, bool TR>
void launch_rot(const SwBandArgs& a, cudaStream_t st) {
  constexpr int NG = 32 / G;
  const size_t smem = 640 + (size_t)kRotWarps * 32 * kLaneProf + (size_t)kRotWarps * NG * kWalkWindow * 8;
  static bool configured = false;
  if (!configured) {
    DRG_CUDA(cudaFuncSetAttribute(k_sw_rot<G, TR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = true;
  }
  const int blocks = ceil_div((long long)(a.hi - a.lo), kRotWarps * NG);
  count_launch();
  k_sw_rot<G, TR><<<blocks, kRotWarps * 32, smem, st>>>(a);
  DRG_CUDA(cudaGetLastError());
}

size_t sw_band_smem(int max_width) {
  const size_t xwords = (size_t)(max_width + kRows + 2) & ~(size_t)1;
  return 640 + (size_t)kBandWarps * 32 * kLaneProf + (size_t)kBandWarps * 2 * xwords * 4;
}

void launch_sw_band(SwBandArgs a, int max_width, bool trace, cudaStream_t st) {
  if (a.hi <= a.lo) return;
  a.xbuf_words = (uint32_t)(((size_t)(max_width + kRows + 2)) & ~(size_t)1);
  const size_t smem = sw_band_smem(max_width);
  static int configured[2] = {0, 0};
  if ((int)smem > configured[trace]) {
    if (trace) DRG_CUDA(cudaFuncSetAttribute(k_sw_band<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else DRG_CUDA(cudaFuncSetAttribute(k_sw_band<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured[trace] = (int)smem;
  }
  const int blocks = ceil_div((long long)(a.hi - a.lo), kBandWarps);
  count_launch();
  if (trace) k_sw_band<true><<<blocks, kBandWarps * 32, smem, st>>>(a);
  else k_sw_band<false><<<blocks, kBandWarps * 32, smem, st>>>(a);
  DRG_CUDA(cudaGetLastError());
}

void launch_sw_band_route(const SwBandArgs& a, int route, int max_width, bool trace, cudaStream_t st) {
  if (a.hi <= a.lo) return;
  switch (route) {
    case 0: trace ? launch_rot<8, true>(a, st) : launch_rot<8, false>(a, st); break;
    case 1: trace ? launch_rot<16, true>(a, st) : launch_rot<16, false>(a, st); break;
    case 2: trace ? launch_rot<32, true>(a, st) : launch_rot<32, false>(a, st); break;
    default: launch_sw_band(a, max_width, trace, st); break;
  }
}

}  // namespace drg
