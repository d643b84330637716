// Integer-pipe issue-rate probe: the roofline denominator of the DP kernel.
// Eight independent chains of s16x2 DPX add-max per thread, one resident
// wave of blocks, timed with CUDA events; the SM clock comes from clock64().
#include "kernels.h"

namespace drg {

namespace {
constexpr int kIters = 4096, kChains = 8;
__global__ void k_probe(uint32_t seed, uint32_t* sink, long long* cycles) {
  uint32_t a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = seed * (threadIdx.x + 1) + k * 0x9E37u;
  long long t0 = clock64();
  unsigned long long g0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(g0));
  for (int it = 0; it < kIters; ++it) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = __viaddmax_s16x2(a[k], a[(k + 1) & (kChains - 1)], seed + k);
  }
  long long t1 = clock64();
  unsigned long long g1;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(g1));
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s ^= a[k];
  if (s == 0x2468ACE1u) sink[0] = s;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    cycles[0] = t1 - t0;
    cycles[1] = (long long)(g1 - g0);  // nanoseconds
  }
}
}  // namespace

void run_int_probe(double* lane_ops_per_s, double* mhz, cudaStream_t st) {
  int dev = 0, sms = 0, per_sm = 0;
  DRG_CUDA(cudaGetDevice(&dev));
  DRG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int threads = 256;
  DRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_probe, threads, 0));
  if (per_sm < 1) per_sm = 1;
  const int blocks = sms * per_sm;
  uint32_t* sink = nullptr;
  long long* cyc = nullptr;
  DRG_CUDA(cudaMalloc(&sink, 16));
  DRG_CUDA(cudaMalloc(&cyc, 16));
  cudaEvent_t e0, e1;
  DRG_CUDA(cudaEventCreate(&e0));
  DRG_CUDA(cudaEventCreate(&e1));
  for (int w = 0; w < 20; ++w) k_probe<<<blocks, threads, 0, st>>>(3u, sink, cyc);  // clocks up
  const int reps = 20;
  DRG_CUDA(cudaEventRecord(e0, st));
  for (int r = 0; r < reps; ++r) k_probe<<<blocks, threads, 0, st>>>(3u, sink, cyc);
  DRG_CUDA(cudaEventRecord(e1, st));
  DRG_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  DRG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  long long c[2] = {0, 0};
  DRG_CUDA(cudaMemcpy(c, cyc, 16, cudaMemcpyDeviceToHost));
  double ops = (double)kIters * kChains * threads * (double)blocks * reps;
  *lane_ops_per_s = ops / (ms * 1e-3);
  *mhz = c[1] > 0 ? (double)c[0] / ((double)c[1] * 1e-3) : 0.0;  // cycles per microsecond
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  cudaFree(cyc);
}

}  // namespace drg
