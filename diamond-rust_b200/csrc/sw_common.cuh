// Shared pieces of the packed 16-bit banded Smith-Waterman kernels: the
// s16x2 helpers, the per-thread register state of one 16-row strip and the
// per-lane subject view.  A strip's 16 rows are 8 pairs of 16-bit lanes: pair
// p holds row p at column c (low half) and row p + 8 at column c - 1 (high
// half).
#pragma once
#include <cstdint>

#include "common.cuh"

namespace drg {
namespace sw {

constexpr int kRows = 16;          // rows per strip
constexpr int kPairs = kRows / 2;  // s16x2 pairs
constexpr int kProfStride = 24;    // bytes per residue row of the strip profile
constexpr int kProfBytes = 26 * kProfStride;
constexpr uint32_t kNeg2 = 0xC000C000u;  // (-16384, -16384)

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
__device__ __forceinline__ uint32_t max2_relu(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("max.s16x2.relu %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}
// Maximum of two pairs of non-negative 16-bit integers below 0x7C00 on the
// FMA pipe: such bit patterns are zero, subnormal or finite positive halves,
// ordered like the integers, and max.f16x2 (no flush to zero) returns one of
// its inputs.
__device__ __forceinline__ uint32_t max2_pos_f16(uint32_t a, uint32_t b) {
  uint32_t r;
  asm("max.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
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
  uint32_t r0, r1;   // prefetched residues of the next two columns
};

// Residue of subject index j, or the sentinel off the sequence.
__device__ __forceinline__ uint32_t subject_residue(const Lane& L, int j) {
  return ((unsigned)j < (unsigned)L.m) ? (uint32_t)__ldg(L.s + j) : (uint32_t)kSentinel;
}
// The residue of column c (subject index jbase + c - 1) from the prefetch
// queue, issuing the load of column c + 2 two steps ahead of its use.
__device__ __forceinline__ uint32_t next_residue(Lane& L, int c) {
  const uint32_t ahead = subject_residue(L, L.jbase + c + 1);
  const uint32_t res = L.r0;
  L.r0 = L.r1;
  L.r1 = ahead;
  return res;
}

template <bool TR>
struct Regs {
  uint32_t H[kPairs], Hm[kPairs], F[kPairs];
  uint32_t E7;        // E of pair 7 at the previous step
  uint32_t htop_old;  // top H of the previous step (D operand of pair 0)
  uint32_t res_prev;  // subject residue of the previous column
  uint32_t rowmax[kPairs];            // per row of the strip: max H so far
  uint32_t rowcol[TR ? kPairs : 1];   // trace mode: first column of that max
};

__device__ __forceinline__ int lo16(uint32_t x) { return (int)(int16_t)(x & 0xFFFFu); }
__device__ __forceinline__ int hi16(uint32_t x) { return (int)(int16_t)(x >> 16); }

}  // namespace sw
}  // namespace drg
