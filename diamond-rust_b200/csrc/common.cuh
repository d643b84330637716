// Shared definitions of the drgpu CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "drgpu.h"

namespace drg {

// An error carrying a DRG_ERR_* code; the C ABI turns it into a status.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define DRG_CUDA(call)                                                                              \
  do {                                                                                              \
    cudaError_t e__ = (call);                                                                       \
    if (e__ != cudaSuccess)                                                                         \
      throw ::drg::Error(e__ == cudaErrorMemoryAllocation ? DRG_ERR_OOM : DRG_ERR_CUDA,             \
                         std::string(#call) + ": " + cudaGetErrorString(e__));                      \
  } while (0)

// Residue codes (alphabet.rs:1-20): 0..19 canonical, 20..22 B/J/Z, 23 X, 24 '*'.
constexpr int kAlpha = 25;
// Code the kernels use for positions outside a sequence; it scores kSentinelScore
// against everything so that cells there can never raise a score.
constexpr int kSentinel = 25;
// Constant-memory banks: one per live context, so that contexts searching with
// different presets or matrices at the same time keep separate tables.
constexpr int kConstSlots = 8;
constexpr int kSentinelScore = -64;

#ifdef __CUDACC__
// Adds every lane's v to *p with one atomic per warp.  All 32 lanes of the
// warp must call it (lanes with nothing to add pass 0): one atomic per thread
// on a single counter serialises in L2 at about one per nanosecond.
__device__ __forceinline__ void warp_sum_atomic(unsigned long long* p, unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(p, v);
}
#endif

// Grow-only device allocation owned by a context; contents are not preserved
// on growth.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  void* ensure(size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (bytes > cap) {
      release();
      size_t want = bytes + bytes / 8;
      DRG_CUDA(cudaMalloc(&p, want));
      cap = want;
    }
    return p;
  }
  template <typename T>
  T* as(size_t n) {
    return static_cast<T*>(ensure(n * sizeof(T)));
  }
  void swap(DevBuf& o) {
    std::swap(p, o.p);
    std::swap(cap, o.cap);
  }
};

// Pinned host staging buffer, grow-only.
struct HostBuf {
  void* p = nullptr;
  size_t cap = 0;
  ~HostBuf() {
    if (p) cudaFreeHost(p);
  }
  void* ensure(size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (bytes > cap) {
      if (p) cudaFreeHost(p);
      p = nullptr;
      size_t want = bytes + bytes / 8;
      DRG_CUDA(cudaMallocHost(&p, want));
      cap = want;
    }
    return p;
  }
  template <typename T>
  T* as(size_t n) {
    return static_cast<T*>(ensure(n * sizeof(T)));
  }
};

// Number of kernels this library has launched in this process (all contexts).
uint64_t kernel_launch_count();
void count_launch();

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }
inline int bits_for(uint64_t v) {  // bits needed to store values 0..v
  int b = 0;
  while (b < 64 && (v >> b) != 0) ++b;
  return b;
}

// Seed shapes as the kernels see them (shape.rs:11-20).
constexpr int kMaxShapes = 64;
constexpr int kMaxWeight = 16;
constexpr int kMaxSpan = 256;  // positions are bytes
struct ShapeTable {
  int n;
  uint8_t weight[kMaxShapes];
  uint16_t span[kMaxShapes];  // up to kMaxSpan (256)
  uint8_t pos[kMaxShapes][kMaxWeight];
};

// Parameters of the seed stage for one search.
struct SeedParams {
  uint8_t bucket[32];      // residue -> reduced bucket, 255 = not seedable
  uint64_t size;           // reduction size
  double cut;              // complexity cut (natural log units)
  double lnfact[33];       // ln n!, summed in the reference's order
  int shape_shift;         // seed key = request << request_shift | shape << shape_shift | key
  int request_shift;
  // Complexity test by the product P of the seed's bucket-count factorials
  // (set by upload_seed_params): P <= p_accept[w] passes the cut, P >=
  // p_reject[w] fails it, and in between the reference's double sum decides.
  uint64_t p_accept[kMaxWeight + 1];
  uint64_t p_reject[kMaxWeight + 1];
  int key32;   // size^weight < 2^32 for every shape
  int prod32;  // every weight <= 12 (P < 2^32)
};

}  // namespace drg
