// Traceback of one band through the nibbles of the trace pass, in the
// reference's order and with its stopping rules (gapped.rs:205-279), shared
// by the band kernel (which walks each band as soon as its DP is done) and
// the stand-alone walk.
//
// The walk keeps a window of 8 consecutive trace words (win[x * win_stride]):
// a diagonal run steps to the next lower word, so one window load (four
// 16-byte loads issued together) serves up to 7 steps instead of one
// dependent load per step.  The residues of matched pairs are compared after
// the walk, run by run, off its dependency chain.
#pragma once
#include "kernels.h"

namespace drg {
namespace sw {

constexpr int kWalkWindow = 8;  // trace words a walker holds

__device__ __forceinline__ void walk_band(const WalkEnv& a, uint64_t t, const Band& b, const TraceBand& tb,
                                          const int8_t* mat, uint2* win, int win_stride) {
  ExactOut R;
  R.score = 0;
  R.q_begin = R.q_end = R.s_begin = R.s_end = 0;
  R.identities = R.positives = R.mismatches = R.gap_openings = R.gaps = R.length = 0;
  R.n_ops = 0;
  R.cells = 0;
  if (tb.score < a.exact_below) return;  // not traced here: the exact kernel writes this band
  const uint8_t* q = a.q_letters + a.q_offsets[b.target] + b.q0;
  const uint8_t* s = a.s_letters + a.s_offsets[b.subject];
  const int64_t m = (int64_t)(a.s_offsets[b.subject + 1] - a.s_offsets[b.subject]);
  const int64_t d0 = b.d0, d1 = b.d1, W = tb.width, rf = tb.row_first;
  if (tb.best_i < 1 || tb.best_i > (int64_t)b.n || tb.best_j < 1 || tb.best_j > m) {
    R.score = -1;  // cannot happen for a best this high; reported to the host as an internal error
    a.out[t] = R;
    return;
  }
  R.score = tb.score;
  R.q_end = (uint32_t)tb.best_i;
  R.s_end = (uint32_t)tb.best_j;
  uint8_t* rev = a.rev + a.ops_off[t];
  uint32_t nrev = 0;
  int state = 0;
  int64_t i = tb.best_i, j = tb.best_j;
  bool in_gap = false;
  int64_t wb = -kWalkWindow;  // first word of the window (even: 16-byte aligned loads)
  while (i > 0 && j > 0) {
    int64_t lo = i - d1, hi = i - d0;
    lo = lo < 0 ? 0 : (lo > m ? m : lo);
    hi = hi < 0 ? 0 : (hi > m ? m : hi);
    if (j < lo || j > hi || i < rf) break;
    const int64_t k = (i - rf) >> 4, r = (i - rf) & 15;
    const int64_t c = j - (rf + 16 * k - d1);
    const int64_t it = c + (r >= 8 ? 1 : 0);
    const uint64_t g = tb.trace_off + (uint64_t)(k * (W + 16) + it) * (uint64_t)tb.stride;
    uint2 w;
    if (tb.stride == 1) {
      if ((int64_t)g < wb || (int64_t)g >= wb + kWalkWindow) {
        wb = (int64_t)g >= 6 ? (((int64_t)g - 6) & ~(int64_t)1) : 0;
        const uint4* src = reinterpret_cast<const uint4*>(a.trace + wb);
        const uint4 v0 = src[0], v1 = src[1], v2 = src[2], v3 = src[3];
        win[0 * win_stride] = make_uint2(v0.x, v0.y);
        win[1 * win_stride] = make_uint2(v0.z, v0.w);
        win[2 * win_stride] = make_uint2(v1.x, v1.y);
        win[3 * win_stride] = make_uint2(v1.z, v1.w);
        win[4 * win_stride] = make_uint2(v2.x, v2.y);
        win[5 * win_stride] = make_uint2(v2.z, v2.w);
        win[6 * win_stride] = make_uint2(v3.x, v3.y);
        win[7 * win_stride] = make_uint2(v3.z, v3.w);
      }
      w = win[(g - wb) * win_stride];
    } else {
      w = a.trace[g];
    }
    const uint32_t p = (uint32_t)(r & 7);
    const uint32_t byte = ((p < 4 ? w.x : w.y) >> (8 * (p & 3))) & 0xFFu;
    const uint32_t nib = r >= 8 ? byte >> 4 : byte & 0xFu;
    // the walk reads only trace words: the residues of the matched pairs
    // are compared afterwards, run by run, off its dependency chain
    if (state == 0) {
      const uint32_t ch = nib & 3;
      if (ch == 0) break;
      if (ch == 1) {
        rev[nrev++] = 0;
        in_gap = false;
        --i;
        --j;
      } else {
        state = ch == 2 ? 1 : 2;
      }
    } else if (state == 1) {
      R.gaps++;
      if (!in_gap) {
        R.gap_openings++;
        in_gap = true;
      }
      rev[nrev++] = 1;
      if (((nib >> 2) & 1) == 0) state = 0;
      --i;
    } else {
      R.gaps++;
      if (!in_gap) {
        R.gap_openings++;
        in_gap = true;
      }
      rev[nrev++] = 2;
      if (((nib >> 3) & 1) == 0) state = 0;
      --j;
    }
  }
  R.q_begin = (uint32_t)i;
  R.s_begin = (uint32_t)j;
  R.length = nrev;
  // ops in alignment order, run-length encoded; a match run of cnt pairs
  // compares q[qi..qi+cnt) with s[sj..sj+cnt) (independent loads)
  uint32_t* o = a.ops + a.ops_off[t];
  uint32_t nops = 0;
  int64_t x = (int64_t)nrev - 1;
  int64_t qi = i, sj = j;  // 0-based positions of the next pair
  while (x >= 0) {
    const uint32_t op = rev[x];
    uint32_t cnt = 0;
    while (x >= 0 && rev[x] == op) {
      ++cnt;
      --x;
    }
    o[nops++] = (cnt << 2) | op;
    if (op == 0) {
      uint32_t ident = 0, pos = 0;
#pragma unroll 4
      for (uint32_t k = 0; k < cnt; ++k) {
        const uint32_t qa = q[qi + k], sb = s[sj + k];
        ident += qa == sb;
        pos += mat[(qa < 24 ? qa : 24) * 25 + (sb < 24 ? sb : 24)] > 0;
      }
      R.identities += ident;
      R.mismatches += cnt - ident;
      R.positives += pos;
      qi += cnt;
      sj += cnt;
    } else if (op == 1) {
      qi += cnt;
    } else {
      sj += cnt;
    }
  }
  R.n_ops = nops;
  a.out[t] = R;
}

}  // namespace sw
}  // namespace drg
