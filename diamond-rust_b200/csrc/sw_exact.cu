// Exact banded Smith-Waterman with traceback (gapped.rs:67-280), one thread
// per band.  It evaluates the reference's recurrence cell by cell in the
// reference's order -- per-row ranges clamped to the subject (gapped.rs:82-96),
// out-of-band H counting as 0 on the diagonal step and E/F starting at the
// band edges, strict comparisons for every tie -- so scores, the first
// row-major maximum, trace bits and the traceback walk are the reference's.
// It runs on the HSPs that survive the E-value gate and the per-query cut,
// and on the rare bands the packed score kernel does not take (width < 17,
// possible 16-bit overflow, best score not above the matrix's largest).
#include "kernels.h"

namespace drg {

namespace {
constexpr int32_t kNeg = INT32_MIN / 4;

__device__ __forceinline__ int64_t clamp64(int64_t v, int64_t lo, int64_t hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

struct MatArg {
  int8_t s[628];
};

__device__ __forceinline__ int sc(const MatArg& M, uint32_t a, uint32_t b) {
  a = a < 24 ? a : 24;
  b = b < 24 ? b : 24;
  return M.s[a * 25 + b];
}

__global__ void k_sw_exact(const ExactJob* __restrict__ jobs, uint64_t n_jobs, int go, int ge, bool trace,
                           uint8_t* __restrict__ scratch, uint32_t* __restrict__ ops_out,
                           ExactOut* __restrict__ out, MatArg M) {
  uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (t >= n_jobs) return;
  const ExactJob J = jobs[t];
  ExactOut R;
  R.score = 0;
  R.q_begin = R.q_end = R.s_begin = R.s_end = 0;
  R.identities = R.positives = R.mismatches = R.gap_openings = R.gaps = R.length = 0;
  R.n_ops = 0;
  R.cells = 0;
  const int64_t n = J.n, m = J.m;
  if (n == 0 || m == 0) {
    out[t] = R;
    return;
  }
  const int64_t d0 = J.d0 < J.d1 ? J.d0 : J.d1;
  const int64_t d1 = J.d0 < J.d1 ? J.d1 : J.d0;
  int64_t wmax = d1 - d0 + 1;
  if (wmax > m + 1) wmax = m + 1;
  uint8_t* base = scratch + J.scratch_off;
  uint64_t trace_bytes = 0;
  if (trace) {
    for (int64_t i = 0; i <= n; ++i) {
      int64_t lo = clamp64(i - d1, 0, m), hi = clamp64(i - d0, 0, m);
      trace_bytes += (uint64_t)(hi - lo + 1);
    }
  }
  uint8_t* tr = base;
  int32_t* rows = reinterpret_cast<int32_t*>(base + ((trace_bytes + 15) & ~15ull));
  int32_t* ph = rows;
  int32_t* pe = rows + wmax;
  int32_t* ch = rows + 2 * wmax;
  int32_t* ce = rows + 3 * wmax;
  const int oc = go + ge;
  // row 0
  int64_t pa = clamp64(-d1, 0, m), pb = clamp64(-d0, 0, m);
  for (int64_t k = 0; k <= pb - pa; ++k) {
    ph[k] = 0;
    pe[k] = kNeg;
  }
  uint64_t off = (uint64_t)(pb - pa + 1);  // trace offset of row 1
  int32_t best = 0;
  int64_t bi = 0, bj = 0;
  uint64_t cells = 0;
  for (int64_t i = 1; i <= n; ++i) {
    const uint32_t qi = J.q[i - 1];
    const int64_t a = clamp64(i - d1, 0, m), b = clamp64(i - d0, 0, m);
    int32_t f_left = kNeg, h_left = kNeg;
    for (int64_t j = a; j <= b; ++j) {
      int32_t d = kNeg;
      if (j >= 1) {
        int32_t hd = (j > pa && j - 1 <= pb) ? ph[j - 1 - pa] : 0;
        d = hd + sc(M, qi, J.s[j - 1]);
      }
      int32_t e = kNeg;
      uint32_t e_ext = 0;
      if (j >= pa && j <= pb) {
        int32_t hp = ph[j - pa];
        if (hp > kNeg / 2 && hp - oc > e) e = hp - oc;
        int32_t pev = pe[j - pa];
        if (pev > kNeg / 2 && pev - ge > e) {
          e = pev - ge;
          e_ext = 1;
        }
      }
      int32_t f = kNeg;
      uint32_t f_ext = 0;
      if (j > a) {
        if (h_left > kNeg / 2 && h_left - oc > f) f = h_left - oc;
        if (f_left > kNeg / 2 && f_left - ge > f) {
          f = f_left - ge;
          f_ext = 1;
        }
      }
      int32_t hv = 0;
      uint32_t choice = 0;
      if (d > hv) { hv = d; choice = 1; }
      if (e > hv) { hv = e; choice = 2; }
      if (f > hv) { hv = f; choice = 3; }
      ch[j - a] = hv;
      ce[j - a] = e;
      if (trace) tr[off + (uint64_t)(j - a)] = (uint8_t)(choice | (e_ext << 2) | (f_ext << 3));
      f_left = f;
      h_left = hv;
      if (hv > best) {
        best = hv;
        bi = i;
        bj = j;
      }
    }
    cells += (uint64_t)(b - a + 1);
    off += (uint64_t)(b - a + 1);
    int32_t* tmp = ph; ph = ch; ch = tmp;
    tmp = pe; pe = ce; ce = tmp;
    pa = a;
    pb = b;
  }
  R.cells = cells;
  if (best <= 0) {
    out[t] = R;
    return;
  }
  R.score = best;
  R.q_end = (uint32_t)bi;
  R.s_end = (uint32_t)bj;
  if (!trace) {
    out[t] = R;
    return;
  }
  // traceback (gapped.rs:205-279); row offsets are rebuilt walking upward.
  uint64_t row_off = off;  // offset of row n + 1
  for (int64_t r = n; r >= bi; --r) {
    int64_t lo = clamp64(r - d1, 0, m), hi = clamp64(r - d0, 0, m);
    row_off -= (uint64_t)(hi - lo + 1);
  }
  // row_off = offset of row bi; reversed single ops go after the row buffers
  uint8_t* rev = reinterpret_cast<uint8_t*>(rows + 4 * wmax);
  uint32_t nrev = 0;
  int state = 0;
  int64_t i = bi, j = bj;
  int64_t ri = bi;  // row whose offset row_off holds
  bool in_gap = false;
  while (i > 0 && j > 0) {
    while (ri > i) {
      --ri;
      int64_t lo = clamp64(ri - d1, 0, m), hi = clamp64(ri - d0, 0, m);
      row_off -= (uint64_t)(hi - lo + 1);
    }
    const int64_t lo = clamp64(i - d1, 0, m), hi = clamp64(i - d0, 0, m);
    if (j < lo || j > hi) break;
    const uint32_t tb = tr[row_off + (uint64_t)(j - lo)];
    if (state == 0) {
      uint32_t c = tb & 3;
      if (c == 0) break;
      if (c == 1) {
        uint32_t x = J.q[i - 1], y = J.s[j - 1];
        R.length++;
        if (x == y) R.identities++;
        else R.mismatches++;
        if (sc(M, x, y) > 0) R.positives++;
        rev[nrev++] = 0;
        in_gap = false;
        --i;
        --j;
      } else {
        state = c == 2 ? 1 : 2;
      }
    } else if (state == 1) {
      R.length++;
      R.gaps++;
      if (!in_gap) {
        R.gap_openings++;
        in_gap = true;
      }
      rev[nrev++] = 1;
      if (((tb >> 2) & 1) == 0) state = 0;
      --i;
    } else {
      R.length++;
      R.gaps++;
      if (!in_gap) {
        R.gap_openings++;
        in_gap = true;
      }
      rev[nrev++] = 2;
      if (((tb >> 3) & 1) == 0) state = 0;
      --j;
    }
  }
  R.q_begin = (uint32_t)i;
  R.s_begin = (uint32_t)j;
  // run-length encode in forward order (the walk produced them reversed)
  uint32_t nops = 0;
  uint32_t* o = ops_out + J.ops_off;
  const uint8_t* tmpb = rev;
  int64_t k = (int64_t)nrev - 1;
  while (k >= 0) {
    uint32_t op = tmpb[k], cnt = 0;
    while (k >= 0 && tmpb[k] == op) {
      ++cnt;
      --k;
    }
    o[nops++] = (cnt << 2) | op;
  }
  R.n_ops = nops;
  out[t] = R;
}
}  // namespace

void launch_sw_exact_with_matrix(const ExactJob* jobs, uint64_t n_jobs, int go, int ge, bool trace,
                                 uint8_t* scratch, uint32_t* ops, ExactOut* out, const int8_t* scores625,
                                 cudaStream_t st) {
  if (n_jobs == 0) return;
  MatArg m;
  for (int i = 0; i < 625; ++i) m.s[i] = scores625[i];
  count_launch();
  k_sw_exact<<<ceil_div(n_jobs, 64), 64, 0, st>>>(jobs, n_jobs, go, ge, trace, scratch, ops, out, m);
  DRG_CUDA(cudaGetLastError());
}

}  // namespace drg
