// Banded affine Smith-Waterman, score only (gapped.rs:67-203), for bands of
// equal width W that share a query window.
//
// Mapping (inter-task): one thread = one band; one warp = up to 32 bands of
// the same query window, so the query profile is shared per warp.  The band is
// swept in strips of 16 DP rows.  Inside a strip, relative column c covers
// absolute subject column j = i0 - d1 + c, and row r of the strip is in the
// band for r <= c <= r + W - 1.  The 16 rows are held as 8 pairs of signed
// 16-bit lanes (DPX s16x2 instructions): pair p holds row p at column c in
// its low half and row p + 8 at column c - 1 in its high half.  With that
// one-column skew every dependency of a pair is already computed:
//   D(i,j) = H(i-1,j-1) + S     previous step of the pair above
//   E(i,j) = max(E(i-1,j) - ge, H(i-1,j) - oc)    this step, pair above
//   F(i,j) = max(F(i,j-1) - ge, H(i,j-1) - oc)    previous step, same pair
//   H      = max(0, D, E, F)
// Row 8's "pair above" is row 7, taken from the previous step; row 0's is the
// previous strip's last row, kept in a per-thread ring in shared memory.
//
// Exactness: values equal the reference's int32 DP while the band's best is
// below 2^15 (bands that could exceed it go to the exact kernel).  Cells with
// j < 0, j > m or rows past the query read a sentinel residue scoring -64;
// they can neither raise the maximum above the true band maximum (when that is
// >= 12; smaller results are recomputed exactly) nor feed an in-band cell.
// Cells left or right of the band in the first/last 16 steps of a strip are
// masked: their H does not count and they pass -inf-like E/F to the band.
#include "kernels.h"

namespace drg {

namespace {

constexpr int kRows = 16;          // rows per strip
constexpr int kPairs = kRows / 2;  // s16x2 pairs
constexpr int kProfStride = 24;    // bytes per residue row of the strip profile
constexpr int kProfBytes = 26 * kProfStride;
constexpr uint32_t kNeg2 = 0xC000C000u;  // (-16384, -16384)
constexpr int kWarpsPerBlock = 4;

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
  return r;
}
__device__ __forceinline__ uint32_t add2(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("add.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
__device__ __forceinline__ uint32_t max2(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("max.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
// keep halves selected by k (0xFFFF per kept half), replace the others with v
__device__ __forceinline__ uint32_t sel2(uint32_t x, uint32_t k, uint32_t v) { return (x & k) | (v & ~k); }

// Sign-extending byte pick: low half = byte b of lo, high half = byte b of hi.
__device__ __forceinline__ constexpr uint32_t pick_sel(int b) {
  return (uint32_t)(b) | ((uint32_t)(8 | b) << 4) | ((uint32_t)(4 + b) << 8) | ((uint32_t)(8 | (4 + b)) << 12);
}

struct Lane {
  const uint8_t* s;  // subject letters
  int m;             // subject length
  int jbase;         // absolute column of relative column 0 in this strip
};

struct Regs {
  uint32_t H[kPairs], Hm[kPairs], F[kPairs];
  uint32_t E7;       // E of pair 7 at the previous step
  uint32_t htop_old; // top H of the previous step (D operand of pair 0)
  uint32_t best;
  uint32_t res_prev; // subject residue of the previous column
};

// One column step.  MODE 0: middle (all rows in band), 1: prologue step
// C (= c), 2: epilogue step C (= c - W).  Masks are compile-time constants.
template <int MODE, int C>
__device__ __forceinline__ void sw_step(Regs& R, const Lane& L, int c, const uint8_t* __restrict__ prof,
                                        uint32_t* __restrict__ ring_r, uint32_t* __restrict__ ring_w, uint32_t noc2,
                                        uint32_t nge2) {
  const int jm1 = L.jbase + c - 1;  // subject index j - 1 of this column
  const uint32_t res = ((unsigned)jm1 < (unsigned)L.m) ? (uint32_t)__ldg(L.s + jm1) : 25u;
  const uint2 lo8 = *reinterpret_cast<const uint2*>(prof + res * kProfStride);
  const uint2 hi8 = *reinterpret_cast<const uint2*>(prof + R.res_prev * kProfStride + 8);
  R.res_prev = res;
  const uint32_t rw = *ring_r;                      // (H, E) of the row above row 0, column c
  const uint32_t htop = prmt(rw, R.H[kPairs - 1], 0x5410);
  uint32_t e_up = prmt(rw, R.E7, 0x5432);
  uint32_t hm_up = add2(htop, noc2);
  uint32_t hd = R.htop_old;
#pragma unroll
  for (int p = 0; p < kPairs; ++p) {
    const uint32_t sc = prmt(p < 4 ? lo8.x : lo8.y, p < 4 ? hi8.x : hi8.y, pick_sel(p & 3));
    const uint32_t d = add2(hd, sc);
    uint32_t e = __viaddmax_s16x2(e_up, nge2, hm_up);
    uint32_t f = __viaddmax_s16x2(R.F[p], nge2, R.Hm[p]);
    uint32_t h = __vimax3_s16x2_relu(d, e, f);
    if (MODE == 1) {
      // left of the band: row p at column C (low), row p+8 at column C-1 (high)
      const bool lo_left = C < p;
      const bool hi_left = C <= p + 8;
      const uint32_t k = (lo_left ? 0u : 0x0000FFFFu) | (hi_left ? 0u : 0xFFFF0000u);
      if (k != 0xFFFFFFFFu) {
        h = h & k;            // no score, H - oc = -oc toward the entry cell
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
    }
    const uint32_t hm = add2(h, noc2);
    R.best = max2(R.best, h);
    hd = R.H[p];
    R.H[p] = h;
    R.Hm[p] = hm;
    R.F[p] = f;
    hm_up = hm;
    e_up = e;
  }
  R.E7 = e_up;
  *ring_w = prmt(R.H[kPairs - 1], R.E7, 0x7632);  // (H, E) of row 15 at column c - 1
  R.htop_old = htop;
}

template <int MODE, int C>
struct Unroll {
  static __device__ __forceinline__ void run(Regs& R, const Lane& L, int c0, const uint8_t* prof, uint32_t* ring,
                                             int buf, int stride, int& slot, uint32_t noc2, uint32_t nge2) {
    int wslot = slot == 0 ? buf - 1 : slot - 1;
    sw_step<MODE, C>(R, L, c0 + C, prof, ring + slot * stride, ring + wslot * stride, noc2, nge2);
    slot = slot + 1 == buf ? 0 : slot + 1;
    Unroll<MODE, C + 1>::run(R, L, c0, prof, ring, buf, stride, slot, noc2, nge2);
  }
};
template <int MODE>
struct Unroll<MODE, kRows> {
  static __device__ __forceinline__ void run(Regs&, const Lane&, int, const uint8_t*, uint32_t*, int, int, int&,
                                             uint32_t, uint32_t) {}
};

__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_sw_score(SwScoreArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t task_id = (uint64_t)blockIdx.x * kWarpsPerBlock + warp;
  const int stride = blockDim.x;
  int8_t* mat = reinterpret_cast<int8_t*>(smem);                        // 25 x 25 scores
  uint8_t* prof = smem + 640 + warp * kProfBytes;                        // strip profile
  uint32_t* ring = reinterpret_cast<uint32_t*>(smem + 640 + kWarpsPerBlock * kProfBytes) + threadIdx.x;
  for (int i = threadIdx.x; i < 625; i += blockDim.x) mat[i] = a.scores625[i];
  __syncthreads();
  if (task_id >= a.n_tasks) return;
  const SwTask task = a.tasks[task_id];
  const int W = (int)task.width;
  const int buf = W + kRows + 1;
  const bool active = lane < (int)task.count;
  const uint32_t bidx = a.order[task.first + (active ? lane : 0)];
  const Band band = a.bands[bidx];
  const uint8_t* q = a.q_letters + a.q_offsets[band.target] + band.q0;
  const int n = (int)band.n;
  Lane L;
  L.s = a.s_letters + a.s_offsets[band.subject];
  L.m = (int)(a.s_offsets[band.subject + 1] - a.s_offsets[band.subject]);
  const uint32_t noc2 = (uint32_t)(uint16_t)(-(a.gap_open + a.gap_extend)) * 0x10001u;
  const uint32_t nge2 = (uint32_t)(uint16_t)(-a.gap_extend) * 0x10001u;
  // ring: boundary row above the first strip is row 0 of the reference (H = 0)
  for (int g = 0; g < buf; ++g) ring[g * stride] = 0xC0000000u;  // H = 0, E = -inf
  int base = 0;  // ring slot of relative column 0 of the current strip
  ring[(W - 1) * stride] = kNeg2;
  Regs R;
  R.best = 0;
  for (uint32_t k = 0; k < task.n_strips; ++k) {
    const int i0 = (int)task.row_first + (int)(k * kRows);
    // strip profile: prof[res * stride + r] = S(q[i0 + r - 1], res)
    __syncwarp();
    for (int e = lane; e < 26 * kRows; e += 32) {
      int res = e >> 4, r = e & 15;
      int i = i0 + r;
      int v;
      if (res == 25 || i > n) v = kSentinelScore;
      else v = mat[(int)min((uint32_t)q[i - 1], 24u) * 25 + res];
      prof[res * kProfStride + r] = (uint8_t)(int8_t)v;
    }
    __syncwarp();
    L.jbase = i0 - band.d1;
#pragma unroll
    for (int p = 0; p < kPairs; ++p) {
      R.H[p] = 0;
      R.Hm[p] = kNeg2;
      R.F[p] = kNeg2;
    }
    R.E7 = kNeg2;
    int slot_m1 = base == 0 ? buf - 1 : base - 1;
    R.htop_old = ring[slot_m1 * stride] & 0xFFFFu;
    R.res_prev = 25u;
    {
      const int jm1 = L.jbase - 2;  // column -1
      R.res_prev = ((unsigned)jm1 < (unsigned)L.m) ? (uint32_t)L.s[jm1] : 25u;
    }
    int slot = base;
    Unroll<1, 0>::run(R, L, 0, prof, ring, buf, stride, slot, noc2, nge2);
    for (int c = kRows; c < W; ++c) {
      int wslot = slot == 0 ? buf - 1 : slot - 1;
      sw_step<0, 0>(R, L, c, prof, ring + slot * stride, ring + wslot * stride, noc2, nge2);
      slot = slot + 1 == buf ? 0 : slot + 1;
    }
    Unroll<2, 0>::run(R, L, W, prof, ring, buf, stride, slot, noc2, nge2);
    // slot now indexes column W + 16 - 1 + 1; column W + 15 of this strip is the
    // next strip's column W - 1: its E/H must read as outside the band.
    int last = slot == 0 ? buf - 1 : slot - 1;
    ring[last * stride] = kNeg2;
    base += kRows;
    if (base >= buf) base -= buf;
  }
  if (active) {
    int lo = (int)(int16_t)(R.best & 0xFFFFu), hi = (int)(int16_t)(R.best >> 16);
    a.score[bidx] = lo > hi ? lo : hi;
  }
}

}  // namespace

size_t launch_sw_score(const SwScoreArgs& a, cudaStream_t st) {
  if (a.n_tasks == 0) return 0;
  const int threads = kWarpsPerBlock * 32;
  const int buf = a.max_width + kRows + 1;
  size_t smem = 640 + kWarpsPerBlock * kProfBytes + (size_t)threads * buf * 4;
  static int configured_max = 0;
  if ((int)smem > configured_max) {
    DRG_CUDA(cudaFuncSetAttribute(k_sw_score, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured_max = (int)smem;
  }
  int blocks = ceil_div((long long)a.n_tasks, kWarpsPerBlock);
  count_launch();
  k_sw_score<<<blocks, threads, smem, st>>>(a);
  DRG_CUDA(cudaGetLastError());
  return smem;
}

}  // namespace drg
