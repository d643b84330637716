// Banded affine Smith-Waterman (gapped.rs:67-203) for many bands that share a
// query window (or a subject, transposed): the score pass of the E-value gate.
//
// Mapping (inter-task): one thread = one band; one warp = up to 32 bands of
// the same query window and width W, so the query profile is shared per warp.
// The band is swept in strips of 16 DP rows.  Inside a strip, relative column
// c covers absolute subject column j = i0 - d1 + c, and row r of the strip is
// in the band for r <= c <= r + W - 1.  The 16 rows are held as 8 pairs of
// signed 16-bit lanes (DPX s16x2 instructions): pair p holds row p at column c
// in its low half and row p + 8 at column c - 1 in its high half.  With that
// one-column skew every dependency of a pair is already computed:
//   D(i,j) = H(i-1,j-1) + S                        previous step, pair above
//   E(i,j) = max(E(i-1,j) - ge, H(i-1,j) - oc)      this step, pair above
//   F(i,j) = max(F(i,j-1) - ge, H(i,j-1) - oc)      previous step, same pair
//   H      = max(0, D, E, F)
// Row 8's "pair above" is row 7, taken from the previous step; row 0's is the
// previous strip's last row, kept in a per-thread ring in shared memory.  The
// ring holds W + 1 words (H - oc | E << 16): a strip reads the previous
// strip's word for column c and then overwrites the slot of column c - 1,
// which is the word the next strip needs at its column c - 17.
//
// A pair update is five half-rate DPX/PRMT operations and one full-rate max:
//   sc = the pair's two scores (one byte permute)
//   F  = max(F - ge, H - oc)            (viaddmax)
//   X  = max(D, F, 0)                   (viaddmax.relu: D = Hdiag + sc fused)
//   E  = max(E - ge, H - oc)            (viaddmax, the step's vertical chain)
//   H  = max(X, E)                      (max.s16x2, full rate)
//   H - oc                              (add, shared by the next E and F)
// Pair 0's diagonal operand comes from the ring and row 7 in the H - oc form
// (that is what the ring keeps), so the profile rows 0 and 8 carry + oc.
//
// Exactness: values equal the reference's int32 DP while the band's best is
// below 31744 = 0x7C00 (bands that could reach it are not given to this
// kernel); the strip maximum relies on that bound (max2_pos_f16).
// Cells with j < 0, j > m or rows past the query read a sentinel residue
// scoring -64; they can neither raise the maximum above the true band maximum
// nor feed an in-band cell.  Rows past m + d1 are not computed: the reference
// keeps one cell per such row, clamped to column m, whose H is at most
// max(largest matrix score, band best - open), so a packed best above the
// matrix's largest score is the reference's; smaller results are recomputed
// exactly.  Cells left or right of the band in the first/last 16 steps of
// a strip are masked: their H does not count and they pass -inf-like E/F.
//
// The traceback of the HSPs that pass the gate runs in sw_band.cu (one warp
// per band) and sw_walk.cuh.
#include "kernels.h"
#include "sw_common.cuh"

namespace drg {

namespace {

using namespace sw;

// Registers of one lane's 16-row strip in the score pass.
struct SRegs {
  uint32_t H[kPairs], Hm[kPairs], F[kPairs];
  uint32_t E7;        // E of pair 7 at the previous step
  uint32_t hmtop_old; // H - oc above pair 0 at the previous step (its D operand, profile + oc)
  const uint8_t* prow_prev;  // profile row of the previous column's residue
  uint32_t mx0, mx1;  // maximum H of the strip so far, folded over rows
};

// One column step.  MODE 0: middle (all rows in band), 1: prologue step
// C (= c), 2: epilogue step C (= c - W) of a warp whose bands share one
// width, 3: step past the narrowest band of a warp with mixed widths
// (cw = c - this lane's W, masks computed at run time).  rp holds the
// (H - oc, E) word of the row above row 0 at column c; wp receives row 15's
// word of column c - 1.
template <int MODE, int C>
__device__ __forceinline__ void sw_step(SRegs& R, Lane& L, int c, const uint8_t* __restrict__ prof,
                                        const uint32_t* __restrict__ rp, uint32_t* __restrict__ wp, uint32_t noc2,
                                        uint32_t nge2, int cw = 0) {
  const uint32_t res = next_residue(L, c);  // subject residue of this column
  const uint8_t* prow = prof + res * kProfStride;
  const uint2 lo8 = *reinterpret_cast<const uint2*>(prow);
  const uint2 hi8 = *reinterpret_cast<const uint2*>(R.prow_prev + 8);
  R.prow_prev = prow;
  const uint32_t rw = *rp;  // (H - oc, E) of the row above row 0, column c
  const uint32_t hm_top = prmt(rw, R.Hm[kPairs - 1], 0x5410);
  uint32_t hm_up = hm_top;
  uint32_t e_up = prmt(rw, R.E7, 0x5432);
  uint32_t hd = R.hmtop_old;
#pragma unroll
  for (int p = 0; p < kPairs; ++p) {
    // Pairs whose two halves are both outside the band at this compile-time
    // step are not computed: left of it in the prologue (C < p), right of it
    // in a one-width epilogue (C >= p + 9).  They take the values the masks
    // below would give (H = 0, H - oc = -oc, F = -inf) and hand the next
    // pair the same E/H the masked computation would; in the prologue every
    // pair below is skipped too, and the E of pair 7 is first read by row 8
    // at step 9, when pair 7 is computed again.
    if ((MODE == 1 && C < p) || (MODE == 2 && C >= p + 9)) {
      hd = R.H[p];
      R.H[p] = 0;
      R.Hm[p] = noc2;
      R.F[p] = kNeg2;
      hm_up = noc2;
      e_up = kNeg2;
      continue;
    }
    const uint32_t sc = prmt(p < 4 ? lo8.x : lo8.y, p < 4 ? hi8.x : hi8.y, pick_sel(p & 3));
    uint32_t f = __viaddmax_s16x2(R.F[p], nge2, R.Hm[p]);
    const uint32_t x = __viaddmax_s16x2_relu(hd, sc, f);  // max(D, F, 0)
    uint32_t e = __viaddmax_s16x2(e_up, nge2, hm_up);
    uint32_t h = max2(x, e);
    if (MODE == 1) {
      // left of the band: row p at column C (low), row p+8 at column C-1 (high)
      const bool lo_left = C < p;
      const bool hi_left = C <= p + 8;
      const uint32_t k = (lo_left ? 0u : 0x0000FFFFu) | (hi_left ? 0u : 0xFFFF0000u);
      if (k != 0xFFFFFFFFu) {
        h = h & k;  // no score; H - oc = -oc toward the entry cell
        f = sel2(f, k, kNeg2);
      }
    } else if (MODE == 2) {
      const bool lo_right = C >= p;
      const bool hi_right = C >= p + 9;
      const uint32_t k = (lo_right ? 0u : 0x0000FFFFu) | (hi_right ? 0u : 0xFFFF0000u);
      if (k != 0xFFFFFFFFu) {
        h = h & k;
        e = sel2(e, k, kNeg2);
      }
    } else if (MODE == 3) {
      // right of this lane's band: row p at column c (low), row p+8 at column c-1 (high)
      const uint32_t k = (cw >= p ? 0u : 0x0000FFFFu) | (cw >= p + 9 ? 0u : 0xFFFF0000u);
      h = h & k;
      e = sel2(e, k, kNeg2);
    }
    const uint32_t hm = add2(h, noc2);
    hd = R.H[p];
    R.H[p] = h;
    R.Hm[p] = hm;
    R.F[p] = f;
    hm_up = hm;
    e_up = e;
  }
  // the strip's maximum, two accumulators of four pairs each, on the FMA
  // pipe (H is in [0, 0x7C00): see max2_pos_f16), beside the ALU's DP work
  R.mx0 = max2_pos_f16(R.mx0, max2_pos_f16(R.H[0], R.H[1]));
  R.mx1 = max2_pos_f16(R.mx1, max2_pos_f16(R.H[4], R.H[5]));
  R.mx0 = max2_pos_f16(R.mx0, max2_pos_f16(R.H[2], R.H[3]));
  R.mx1 = max2_pos_f16(R.mx1, max2_pos_f16(R.H[6], R.H[7]));
  R.E7 = e_up;
  *wp = prmt(R.Hm[kPairs - 1], R.E7, 0x7632);  // (H - oc, E) of row 15 at column c - 1
  R.hmtop_old = hm_top;
}

// The ring of one lane: W + 1 words at stride `stride`; rp reads column c,
// wp (the slot read one step earlier) takes column c - 1.
struct RingPtr {
  uint32_t *rp, *wp;
  uint32_t* begin;
  uint32_t* end;
  int stride;
  __device__ __forceinline__ void advance() {
    wp = rp;
    rp += stride;
    if (rp == end) rp = begin;
  }
};

template <int MODE, int C>
struct Unroll {
  static __device__ __forceinline__ void run(SRegs& R, Lane& L, int c0, const uint8_t* prof, RingPtr& rg,
                                             uint32_t noc2, uint32_t nge2) {
    sw_step<MODE, C>(R, L, c0 + C, prof, rg.rp, rg.wp, noc2, nge2);
    rg.advance();
    Unroll<MODE, C + 1>::run(R, L, c0, prof, rg, noc2, nge2);
  }
};
template <int MODE>
struct Unroll<MODE, kRows> {
  static __device__ __forceinline__ void run(SRegs&, Lane&, int, const uint8_t*, RingPtr&, uint32_t, uint32_t) {}
};

// Score pass: scores[band] = the band's best H, best_row[band] = the last row
// of the first strip that holds it (an upper bound of the reference's best_i,
// which is all the traceback pass needs).
// Shared memory holds three blocks per SM in the 4- and 2-warp classes, so
// registers are budgeted for three (without the hint the compiler spills).
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32, WARPS >= 2 ? 3 : 1) k_sw(SwScoreArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t task_id = a.task_lo + (uint64_t)blockIdx.x * WARPS + warp;
  const int stride = WARPS * 32;
  int8_t* mat = reinterpret_cast<int8_t*>(smem);  // 25 x 25 scores
  uint8_t* prof = smem + 640 + warp * kProfBytes;  // strip profile
  uint32_t* ring = reinterpret_cast<uint32_t*>(smem + 640 + WARPS * kProfBytes) + threadIdx.x;
  for (int i = threadIdx.x; i < 625; i += blockDim.x) mat[i] = a.scores625[i];
  __syncthreads();
  if (task_id >= a.task_hi) return;
  const SwTask task = a.tasks[task_id];
  const int W = (int)task.width;   // widest band of the warp
  const int Wmin = (int)task.w_min;
  const int buf = W + 1;
  const bool active = lane < (int)task.count;
  const uint32_t bidx = a.order[task.first + (active ? lane : 0)];
  const Band band = a.bands[bidx];
  const int Wl = band.d1 - band.d0 + 1;  // this lane's width
  // Rows are the query window and columns the subject, or (a transposed
  // task, whose lanes share the subject) rows the subject and columns the
  // window with the diagonals negated: the same cells, so the same best.
  const bool tr = task.transposed != 0;
  const uint8_t* qw = a.q_letters + a.q_offsets[band.target] + band.q0;
  const uint8_t* sj = a.s_letters + a.s_offsets[band.subject];
  const int m_s = (int)(a.s_offsets[band.subject + 1] - a.s_offsets[band.subject]);
  const uint8_t* q = tr ? sj : qw;  // row letters
  const int n = tr ? m_s : (int)band.n;
  const int d1 = tr ? -band.d0 : band.d1;
  Lane L;
  L.s = tr ? qw : sj;  // column letters
  L.m = tr ? (int)band.n : m_s;
  const int oc = a.gap_open + a.gap_extend;  // at most kSwMaxOpenCost (profile bytes carry it)
  const uint32_t noc2 = (uint32_t)(uint16_t)(-oc) * 0x10001u;
  const uint32_t nge2 = (uint32_t)(uint16_t)(-a.gap_extend) * 0x10001u;
  // dead cell word: H = 0 (H - oc = -oc), E = -inf
  const uint32_t dead = 0xC0000000u | (noc2 & 0xFFFFu);
  // the row above the first strip is row 0 of the reference: H = 0, and its
  // E is -inf; column Wl - 1 is outside row 0's band on the right.
  for (int g = 0; g < buf; ++g) ring[g * stride] = dead;
  ring[(Wl - 1) * stride] = kNeg2;
  RingPtr rg;
  rg.begin = ring;
  rg.end = ring + buf * stride;
  rg.stride = stride;
  int base = 0;  // ring slot of relative column 0 of the current strip
  SRegs R;
  int best = 0, best_i = 0;
  uint64_t steps_done = 0;  // column steps run (all strips)
  for (uint32_t k = 0; k < task.n_strips; ++k) {
    const int i0 = (int)task.row_first + (int)(k * kRows);
    // strip profile: prof[res * stride + r] = S(query letter, subject letter)
    // of row i0 + r against column residue res, + oc in rows 0 and 8 (their
    // diagonal operand is H - oc)
    __syncwarp();
    for (int e = lane; e < 26 * kRows; e += 32) {
      int res = e >> 4, r = e & 15;
      int i = i0 + r;
      int v;
      if (res == 25 || i > n) v = kSentinelScore;
      else {
        const int row = (int)min((uint32_t)q[i - 1], 24u);
        v = tr ? mat[res * 25 + row] : mat[row * 25 + res];
      }
      if ((r & 7) == 0) v += oc;
      prof[res * kProfStride + r] = (uint8_t)(int8_t)v;
    }
    __syncwarp();
    L.jbase = i0 - d1;
    // column c_begin - 1 of the strip: dead cells (H = 0, so H - oc = -oc,
    // which is also pair 0's diagonal operand and row 8's E source)
#pragma unroll
    for (int p = 0; p < kPairs; ++p) {
      R.H[p] = 0;
      R.Hm[p] = noc2;
      R.F[p] = kNeg2;
    }
    R.mx0 = R.mx1 = 0;
    R.E7 = kNeg2;
    // Steps whose cells all lie off the matrix for every lane of the warp are
    // skipped: at step c a lane's cells sit at subject columns jbase + c (rows
    // 0-7) and jbase + c - 1 (rows 8-15), all j <= 0 for c <= -jbase and all
    // j > m for c >= m + 2 - jbase.  Such cells are H = 0 on the left and can
    // never exceed an in-matrix value on the right, so only the ring words a
    // later strip reads need care (below).
    const int lead = __reduce_min_sync(0xFFFFFFFFu, max(0, 1 - L.jbase));
    const int trail = __reduce_max_sync(0xFFFFFFFFu, L.m + 2 - L.jbase);
    const int c_begin = lead >= kRows ? min(lead, Wmin) : 0;  // whole prologue or none of it
    const int c_end = max(c_begin, min(W + kRows, max(trail, kRows)));
    steps_done += (uint64_t)(c_end - c_begin);
    {
      int slot = base + c_begin;
      slot = slot >= buf ? slot - buf : slot;
      rg.rp = ring + slot * stride;
      rg.wp = ring + (slot == 0 ? buf - 1 : slot - 1) * stride;
    }
    // H - oc of column c_begin - 1 of the row above; row 7 not yet computed: H = 0
    R.hmtop_old = (*rg.wp & 0xFFFFu) | (noc2 & 0xFFFF0000u);
    {
      const int jm1 = L.jbase + c_begin - 2;  // column c_begin - 1
      R.prow_prev = prof + subject_residue(L, jm1) * kProfStride;
      L.r0 = subject_residue(L, jm1 + 1);  // columns c_begin and c_begin + 1
      L.r1 = subject_residue(L, jm1 + 2);
    }
    int c = c_begin;
    if (c_begin == 0) {
      Unroll<1, 0>::run(R, L, 0, prof, rg, noc2, nge2);
      c = kRows;
    }
    const int mid_end = min(Wmin, c_end);
    {
      // in runs that end where the read pointer wraps, so that the steps
      // themselves carry no wrap test
      uint32_t* rp = rg.rp;
      uint32_t* wp = rg.wp;
      while (c < mid_end) {
        const int stop = min(mid_end, c + (int)((rg.end - rp) / stride));
#pragma unroll 2
        for (; c < stop; ++c) {
          sw_step<0, 0>(R, L, c, prof, rp, wp, noc2, nge2);
          wp = rp;
          rp += stride;
        }
        if (rp == rg.end) rp = rg.begin;
      }
      rg.rp = rp;
      rg.wp = wp;
    }
    if (Wmin == W && c == W && c_end == W + kRows) {  // one width in the warp: compile-time masks
      Unroll<2, 0>::run(R, L, W, prof, rg, noc2, nge2);
    } else {  // mixed widths or an early stop: each lane masks past its own right edge
      for (; c < c_end; ++c) {
        sw_step<3, 0>(R, L, c, prof, rg.rp, rg.wp, noc2, nge2, c - Wl);
        rg.advance();
      }
    }
    // Ring words the next strip may read that this strip did not write: the
    // next strip's column x reads this strip's column x + 16.  Skipped columns
    // on the left hold dead cells (H = 0, E = -inf); past the early stop the
    // next strip computes only off-matrix cells, which must see -inf.
    for (int x = kRows - 1; x <= c_begin - 2; ++x) {
      int ls = base + x;
      ls = ls >= buf ? ls - buf : ls;
      ring[ls * stride] = dead;
    }
    if (c_end < W + kRows) {
      const int x_hi = min(W + kRows - 1, max(c_end - 1, 2 * kRows - 1));
      for (int x = c_end - 1; x <= x_hi; ++x) {
        int ls = base + x;
        ls = ls >= buf ? ls - buf : ls;
        ls = ls >= buf ? ls - buf : ls;
        ring[ls * stride] = kNeg2;
      }
    }
    // this lane's column Wl + 15 is the next strip's column Wl - 1: outside
    // the band on the right, its E/H must read as -inf.
    {
      int ls = base + Wl + kRows - 1;
      ls = ls >= buf ? ls - buf : ls;
      ls = ls >= buf ? ls - buf : ls;
      ring[ls * stride] = kNeg2;
    }
    base += kRows;
    if (base >= buf) base -= buf;
    // strictly greater: the first strip holding the maximum keeps it
    const uint32_t m2 = max2(R.mx0, R.mx1);
    const int v = max(lo16(m2), hi16(m2));
    if (v > best) {
      best = v;
      best_i = i0 + kRows - 1;
    }
  }
  if (lane == 0 && a.cells_eval) {
    atomicAdd(a.cells_eval, (unsigned long long)(steps_done * kRows * task.count));
    atomicAdd(a.cells_eval + 2, (unsigned long long)(steps_done * kRows * 32));  // idle lanes included
  }
  if (!active) return;
  a.score[bidx] = best;
  // transposed: the best cell's subject row i' <= best_i sits on query row
  // i' + d (d in [d0, d1]), so best_i + d1 bounds the reference's best row
  if (tr && best_i > 0) best_i = min((int)band.n, best_i + band.d1);
  if (a.best_row) a.best_row[bidx] = best_i;
}

template <int WARPS>
void launch_class(const SwScoreArgs& a, int max_width, cudaStream_t st) {
  if (a.task_hi <= a.task_lo) return;
  const int threads = WARPS * 32;
  const size_t smem = 640 + WARPS * kProfBytes + (size_t)threads * (max_width + 1) * 4;
  static int configured = 0;  // per template instance
  if ((int)smem > configured) {
    DRG_CUDA(cudaFuncSetAttribute(k_sw<WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = (int)smem;
  }
  const int blocks = ceil_div((long long)(a.task_hi - a.task_lo), WARPS);
  count_launch();
  k_sw<WARPS><<<blocks, threads, smem, st>>>(a);
  DRG_CUDA(cudaGetLastError());
}

}  // namespace

int sw_width_class(int width) {
  if (width < kSwMinWidth) return -1;
  for (int c = 0; c < kSwClasses; ++c)
    if (width <= kSwClassMax[c]) return c;
  return -1;
}

void launch_sw_class(const SwScoreArgs& a, int cls, cudaStream_t st) {
  switch (cls) {
    case 0: launch_class<4>(a, kSwClassMax[0], st); break;
    case 1: launch_class<2>(a, kSwClassMax[1], st); break;
    case 2: launch_class<1>(a, kSwClassMax[2], st); break;
    default: launch_class<1>(a, kSwClassMax[3], st); break;
  }
}


}  // namespace drg
