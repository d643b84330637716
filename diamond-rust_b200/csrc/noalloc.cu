// gapped::extend_span with traceback for callers that must not allocate.
//
// Some callers cannot call cudaMalloc: services that own every byte of device
// memory through their own pool and forbid allocations by libraries on the
// request path, and real-time loops that may not take the allocator's locks
// or wait for its latency.  drg_extend_span_noalloc gives them the exact
// banded Smith-Waterman (the kernel behind drg_extend_span_batch) with every
// buffer supplied by the caller, and its scratch in a fixed static device
// array:
//
//  - the scratch is g_noalloc_scratch below, 32 MiB, present on every GPU that
//    loads this library until the process exits;
//  - a call whose bands need more than that is rejected (DRG_ERR_INVALID and
//    a message saying how many bytes it needed) before any work is queued;
//  - the first call on a device, with that device current, looks up the
//    array's device address (cudaGetSymbolAddress);
//  - all calls share the one array, so calls whose work overlaps on the GPU
//    (other streams, other host threads) race: order them on one stream or
//    serialise them.  Nothing in the array has to start at zero: a call
//    writes every byte it reads before reading it.
// No cudaMalloc, cudaFree, host heap or library allocation is made here.
#include <mutex>

#include <cub/block/block_scan.cuh>

#include "kernels.h"
#include "host/scoring.h"

namespace drg {

namespace {

constexpr uint64_t kNoAllocScratchBytes = 32ull << 20;
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
uint8_t* g_scratch_address[kMaxDevices] = {};

uint64_t round256(uint64_t x) { return (x + 255) & ~255ull; }

// Device address of g_noalloc_scratch on the current device (host code may
// not use the symbol itself: on the host it names a stand-in, not device memory).
cudaError_t scratch_address(uint8_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_address[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_address[dev] = static_cast<uint8_t*>(p);
  }
  *out = g_scratch_address[dev];
  return cudaSuccess;
}

struct Layout {
  uint64_t jobs, q_off, s_off, exact_jobs, exact_out, dp, total;
};

constexpr int kPrepThreads = 1024;

// One block: the kernel's job descriptors and their scratch and op offsets,
// built from the copies of the caller's host arrays.  Thread t takes a
// contiguous run of jobs, so a block-wide exclusive scan of the threads'
// totals gives each run its first offsets.
__global__ void __launch_bounds__(kPrepThreads) k_noalloc_prepare(const drg_span_job* __restrict__ jobs,
                                                                  uint32_t n_jobs, const uint64_t* __restrict__ q_off,
                                                                  const uint64_t* __restrict__ s_off,
                                                                  const uint8_t* q_letters, const uint8_t* s_letters,
                                                                  ExactJob* __restrict__ out) {
  using Scan = cub::BlockScan<uint64_t, kPrepThreads>;
  __shared__ typename Scan::TempStorage tmp;
  const uint32_t per = (n_jobs + kPrepThreads - 1) / kPrepThreads;
  const uint32_t lo = min(n_jobs, threadIdx.x * per), hi = min(n_jobs, lo + per);
  uint64_t scratch = 0, slots = 0;
  for (uint32_t i = lo; i < hi; ++i) {
    const drg_span_job j = jobs[i];
    ExactJob e;
    e.q = q_letters + q_off[j.query];
    e.s = s_letters + s_off[j.subject];
    e.n = (uint32_t)(q_off[j.query + 1] - q_off[j.query]);
    e.m = (uint32_t)(s_off[j.subject + 1] - s_off[j.subject]);
    e.d0 = (int32_t)j.d0;
    e.d1 = (int32_t)j.d1;
    e.scratch_off = scratch;  // within the thread's run for now
    e.ops_off = slots;
    scratch += exact_scratch_bytes(e.n, e.m, e.d0, e.d1, true);
    slots += (uint64_t)e.n + e.m;
    out[i] = e;
  }
  uint64_t scratch0, slots0;
  Scan(tmp).ExclusiveSum(scratch, scratch0);
  __syncthreads();
  Scan(tmp).ExclusiveSum(slots, slots0);
  for (uint32_t i = lo; i < hi; ++i) {
    out[i].scratch_off += scratch0;
    out[i].ops_off += slots0;
  }
}

__global__ void k_noalloc_finish(const ExactJob* __restrict__ jobs, const ExactOut* __restrict__ eo, uint32_t n,
                                 drg_aligned* __restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const ExactOut r = eo[i];
  drg_aligned a;
  a.found = r.score > 0 ? 1 : 0;
  a.score = r.score > 0 ? r.score : 0;
  a.q_begin = a.found ? r.q_begin : 0;
  a.q_end = a.found ? r.q_end : 0;
  a.s_begin = a.found ? r.s_begin : 0;
  a.s_end = a.found ? r.s_end : 0;
  a.identities = a.found ? r.identities : 0;
  a.positives = a.found ? r.positives : 0;
  a.mismatches = a.found ? r.mismatches : 0;
  a.gap_openings = a.found ? r.gap_openings : 0;
  a.gaps = a.found ? r.gaps : 0;
  a.length = a.found ? r.length : 0;
  a.cells = r.cells;
  a.n_ops = a.found ? r.n_ops : 0;
  a.pad = 0;
  a.ops_offset = jobs[i].ops_off;
  out[i] = a;
}

int fail(char* err, size_t cap, int code, const char* msg, unsigned long long a = 0, unsigned long long b = 0) {
  if (err && cap) snprintf(err, cap, msg, a, b);
  return code;
}

}  // namespace
}  // namespace drg

using namespace drg;

extern "C" int drg_extend_span_noalloc(const uint8_t* d_q_letters, const uint64_t* q_offsets, uint64_t n_q,
                                       const uint8_t* d_s_letters, const uint64_t* s_offsets, uint64_t n_s,
                                       const drg_span_job* jobs, uint64_t n_jobs, const char* matrix,
                                       int32_t gap_open, int32_t gap_extend, drg_aligned* d_out, uint32_t* d_ops,
                                       uint64_t ops_capacity, void* stream, char* err, size_t err_cap) {
  if (!q_offsets || !s_offsets || (n_jobs && (!jobs || !d_out || !d_q_letters || !d_s_letters)))
    return fail(err, err_cap, DRG_ERR_INVALID, "null argument");
  if (n_jobs > (1ull << 20)) return fail(err, err_cap, DRG_ERR_INVALID, "at most %llu jobs per call", 1ull << 20);
  Scoring sc;
  {
    std::string e;
    if (!make_scoring(matrix, gap_open, gap_extend, &sc, &e)) return fail(err, err_cap, DRG_ERR_INVALID,
                                                                          "unknown matrix or gap costs");
  }
  // sizes, from the caller's host arrays only
  uint64_t dp = 0, ops = 0;
  for (uint64_t i = 0; i < n_jobs; ++i) {
    const drg_span_job& j = jobs[i];
    if (j.query >= n_q || j.subject >= n_s) return fail(err, err_cap, DRG_ERR_INVALID, "job %llu: index out of range", i);
    if (j.d0 < INT32_MIN / 2 || j.d0 > INT32_MAX / 2 || j.d1 < INT32_MIN / 2 || j.d1 > INT32_MAX / 2)
      return fail(err, err_cap, DRG_ERR_INVALID, "job %llu: diagonal out of range", i);
    if (q_offsets[j.query + 1] < q_offsets[j.query] || s_offsets[j.subject + 1] < s_offsets[j.subject])
      return fail(err, err_cap, DRG_ERR_INVALID, "job %llu: offsets decrease", i);
    uint64_t n = q_offsets[j.query + 1] - q_offsets[j.query], m = s_offsets[j.subject + 1] - s_offsets[j.subject];
    if (n >= (1ull << 31) || m >= (1ull << 31))
      return fail(err, err_cap, DRG_ERR_INVALID, "job %llu: sequence longer than 2^31 letters", i);
    dp += exact_scratch_bytes((uint32_t)n, (uint32_t)m, (int32_t)j.d0, (int32_t)j.d1, true);
    ops += n + m;
  }
  if (ops > ops_capacity || (ops && !d_ops))
    return fail(err, err_cap, DRG_ERR_INVALID, "op buffer holds %llu entries, the bands need %llu",
                (unsigned long long)ops_capacity, (unsigned long long)ops);
  Layout L;
  L.jobs = 0;
  L.q_off = round256(L.jobs + n_jobs * sizeof(drg_span_job));
  L.s_off = round256(L.q_off + (n_q + 1) * sizeof(uint64_t));
  L.exact_jobs = round256(L.s_off + (n_s + 1) * sizeof(uint64_t));
  L.exact_out = round256(L.exact_jobs + n_jobs * sizeof(ExactJob));
  L.dp = round256(L.exact_out + n_jobs * sizeof(ExactOut));
  L.total = L.dp + dp;
  if (L.total > kNoAllocScratchBytes)
    return fail(err, err_cap, DRG_ERR_INVALID, "call needs %llu bytes of scratch, the static scratch holds %llu",
                (unsigned long long)L.total, (unsigned long long)kNoAllocScratchBytes);
  if (n_jobs == 0) return DRG_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  {
    // the scratch address is the current device's, so the stream must be too
    int cur = 0, sdev = 0;
    cudaError_t ce = cudaGetDevice(&cur);
    if (ce == cudaSuccess) ce = cudaStreamGetDevice(st, &sdev);
    if (ce != cudaSuccess) return fail(err, err_cap, DRG_ERR_CUDA, "cannot query the stream's device (%llu)", ce);
    if (sdev != cur)
      return fail(err, err_cap, DRG_ERR_INVALID, "stream belongs to device %llu, the current device is %llu",
                  (unsigned long long)sdev, (unsigned long long)cur);
  }
  uint8_t* base = nullptr;
  cudaError_t ce = scratch_address(&base);
  if (ce != cudaSuccess) return fail(err, err_cap, DRG_ERR_CUDA, "cudaGetSymbolAddress failed (%llu)", (unsigned long long)ce);
  try {
    DRG_CUDA(cudaMemcpyAsync(base + L.jobs, jobs, n_jobs * sizeof(drg_span_job), cudaMemcpyHostToDevice, st));
    DRG_CUDA(cudaMemcpyAsync(base + L.q_off, q_offsets, (n_q + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    DRG_CUDA(cudaMemcpyAsync(base + L.s_off, s_offsets, (n_s + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    ExactJob* ej = reinterpret_cast<ExactJob*>(base + L.exact_jobs);
    ExactOut* eo = reinterpret_cast<ExactOut*>(base + L.exact_out);
    count_launch();
    k_noalloc_prepare<<<1, kPrepThreads, 0, st>>>(reinterpret_cast<const drg_span_job*>(base + L.jobs), (uint32_t)n_jobs,
                                         reinterpret_cast<const uint64_t*>(base + L.q_off),
                                         reinterpret_cast<const uint64_t*>(base + L.s_off), d_q_letters, d_s_letters,
                                         ej);
    DRG_CUDA(cudaGetLastError());
    launch_sw_exact_with_matrix(ej, n_jobs, sc.gap_open, sc.gap_extend, true, base + L.dp, d_ops, eo, sc.scores, st);
    count_launch();
    k_noalloc_finish<<<ceil_div((long long)n_jobs, 128), 128, 0, st>>>(ej, eo, (uint32_t)n_jobs, d_out);
    DRG_CUDA(cudaGetLastError());
  } catch (const Error& e) {
    return fail(err, err_cap, e.code, "CUDA error while queueing the bands");
  }
  return DRG_OK;
}
