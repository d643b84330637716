// Library objects behind the opaque C handles.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "host/pool.h"
#include "index_cache.h"
#include "drgpu.h"
#include "host/presets.h"
#include "host/scoring.h"

struct drg_ctx {
  int device = 0;
  int slot = -1;                // constant-memory bank of this context (kConstSlots of them)
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;  // concurrent launches (wide-band classes)
  cudaMemPool_t pool = nullptr;  // resident databases and batches (kept across calls)
  std::string err;
  // seed stage
  drg::DevBuf q_keys, q_vals, q_keys_s, q_vals_s, r_keys, r_vals, r_keys_s, r_vals_s, cub_tmp;
  drg::DevBuf run_keys, run_keys32, run_counts, run_qstart, run_rlo, run_rcount, run_hits, run_hit_off, counters;
  drg::DevBuf q_owner, r_owner, seed_filter, seed_counts, ref_first, hit_coarse, target_hits, run_qlo, run_qcount;
  // hits and ungapped stage
  drg::DevBuf hits, hits_s, hits_u, flags, idx, segs, seg_keys, segs_c, keep;
  // bands and DP
  drg::DevBuf bands, bands_c, band_valid, pair_first, sw_keys, sw_keys_s, sw_order, sw_order_s, sw_tasks, scores,
      state, sel_idx, sel_bands, exact_jobs, exact_out, exact_scratch, exact_ops;
  drg::DevBuf tband, task_size, task_off, trace, rev, ex_bands, ops_off, trace_out, task_max;
  drg::DevBuf sw_tasks_u, task_key, task_key_s, task_val, task_val_s, best_row, band_jobs_u, band_jobs, sw_rows, sw_rows_s,
      sw_keys_r, sw_order_r;
  drg::DevBuf bj_key, bj_key_s, bj_val, bj_val_s, bj_size, bj_off, bj_max, ops_cnt, ops_coff, ops_compact, verdict,
      tr_count, letter_check;
  // blastx front end
  drg::DevBuf x_nt, x_nt_off, x_len, x_scratch_off, x_scratch, x_keep, x_kept_len, x_kept_index, x_kept_off,
      x_query, x_frame;
  drg::DevBuf pass_counts, sw_counts;             // device-side counts of one pass of the stages after the join
  drg::SortScratch sort_tmp;
  drg::SortScratch sort_tmp_side;  // a sort on the side stream beside one on the main stream
  drg::DevBuf sort_err;  // radix sort scratch; its wait-timeout word (checked after the work)
  drg_tuning tuning{273, 17, 1, 0};  // tile and routing choices (include/drgpu.h)
  drg::HostBuf h_stage;
  cudaEvent_t ev[16] = {};
  drg_run_stats last{};
  std::unique_ptr<drg::host::Pool> host_pool;  // CPU-side steps of a search, created on first use
};

struct drg_db {
  drg_ctx* ctx = nullptr;
  uint8_t* letters = nullptr;   // device, 16 bytes of slack after the end
  uint8_t* score_letters = nullptr;  // device: letters clamped to 24, only when some code is above 24
  uint64_t* offsets = nullptr;  // device, n + 1
  uint32_t* owner = nullptr;    // device: letter -> sequence
  std::vector<uint64_t> h_offsets;
  uint64_t n = 0, total = 0;
  uint32_t max_len = 0;
  std::unique_ptr<drg::IndexCache> cache;  // sorted reference seeds kept for later searches
};

struct drg_batch {
  drg_ctx* ctx = nullptr;
  uint8_t* letters = nullptr;
  uint8_t* score_letters = nullptr;  // device: letters clamped to 24, only when some code is above 24
  uint64_t* offsets = nullptr;
  uint32_t* owner = nullptr;
  uint32_t* request = nullptr;  // device: request of each target (null: one request)
  uint32_t max_request = 0;     // largest request id (the seed keys' request field width)
  std::vector<uint64_t> h_offsets;
  std::vector<uint32_t> query;
  std::vector<uint8_t> frame;
  uint64_t n = 0, total = 0;
  uint32_t max_len = 0;
};

namespace drg {
struct Band;
// Device sequences: letters + offsets (device) and the host copy of offsets.
struct DevSeqs {
  const uint8_t* letters;
  const uint64_t* offsets;
  const std::vector<uint64_t>* h_offsets;
  const uint8_t* score_letters = nullptr;  // letters clamped to 24, when some code is above 24
  // what the DP kernels read: they index residue profiles by the code
  const uint8_t* dp_letters() const { return score_letters ? score_letters : letters; }
};
// Stage times of a search without draining the stream: spans between
// recorded events, read once the work has been waited for (resolve()).
class TimeLog {
 public:
  TimeLog() = default;
  TimeLog(const TimeLog&) = delete;
  TimeLog& operator=(const TimeLog&) = delete;
  ~TimeLog() {
    for (cudaEvent_t e : events_) cudaEventDestroy(e);
  }
  // A new event owned by the log (the caller records it).
  cudaEvent_t event() {
    cudaEvent_t e;
    DRG_CUDA(cudaEventCreate(&e));
    events_.push_back(e);
    return e;
  }
  // *dst += milliseconds from a to b, at resolve().
  void span(cudaEvent_t a, cudaEvent_t b, double* dst) { spans_.push_back({a, b, dst}); }
  // f runs at resolve(), after the spans.
  void later(std::function<void()> f) { jobs_.push_back(std::move(f)); }
  // Every event recorded so far must have completed.
  void resolve() {
    for (const Span& s : spans_) {
      float ms = 0;
      DRG_CUDA(cudaEventElapsedTime(&ms, s.a, s.b));
      *s.dst += ms;
    }
    for (auto& f : jobs_) f();
    spans_.clear();
    jobs_.clear();
  }

 private:
  struct Span {
    cudaEvent_t a, b;
    double* dst;
  };
  std::vector<cudaEvent_t> events_;
  std::vector<Span> spans_;
  std::vector<std::function<void()>> jobs_;
};

struct ExactOut;
// With a TimeLog the kernel times go into it; without one they are read
// before returning (which waits for the launches).
void run_bands(drg_ctx* c, const Band* bands, uint64_t n_bands, const DevSeqs& q, const DevSeqs& s,
               const Scoring& sc, bool trace, int32_t* scores, int32_t* best_row, ExactOut* out, uint32_t* ops,
               const uint64_t* d_ops_off, const std::vector<uint64_t>* h_ops_off, drg_run_stats& st,
               int64_t* d_count, unsigned long long* cells_gpu, TimeLog* times = nullptr);
// Whole-path search over resident inputs (pipeline.cu).
void search(drg_ctx* ctx, const drg_db* db, const drg_batch* b, const drg_search_config* cfg, drg_result* out);
// Whether n device letters hold a code above 24; syncs the context's stream.
bool letters_above_24(drg_ctx* ctx, const uint8_t* d_letters, uint64_t n);
// Device residency helpers.
drg_db* make_db(drg_ctx* ctx, const uint8_t* letters, const uint64_t* offsets, uint64_t n);
drg_batch* make_batch(drg_ctx* ctx, const uint8_t* letters, const uint64_t* offsets, const uint32_t* query,
                      const uint8_t* frame, uint64_t n, const uint32_t* request = nullptr);
// blastx targets translated on the device from host reads; with `host`, the
// frames are also returned (letters, offsets, query index, frame).
struct HostFrames {
  std::vector<uint8_t> letters;
  std::vector<uint64_t> offsets;
  std::vector<uint32_t> query;
  std::vector<uint8_t> frame;
};
drg_batch* make_batch_translated(drg_ctx* ctx, const uint8_t* nt, const uint64_t* nt_offsets, uint64_t n_reads,
                                 int64_t min_orf, HostFrames* host = nullptr);
void free_db(drg_db* db);
void free_batch(drg_batch* b);
}  // namespace drg
