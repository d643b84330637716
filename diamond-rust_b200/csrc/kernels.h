// Launch wrappers of the drgpu kernels (host-callable, stream-ordered).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"

namespace drg {

// ---- seeds (seed_kernels.cu) ----------------------------------------------
// Shape table and seed parameters into constant bank `slot` (the context's).
void upload_seed_params(const ShapeTable& shapes, const SeedParams& p, int slot, cudaStream_t st);
// seq index of every letter: out[g] = i with offsets[i] <= g < offsets[i+1].
void launch_letter_owner(const uint64_t* offsets, uint64_t n_seqs, uint64_t letter_lo, uint64_t letter_hi,
                         uint32_t* out, cudaStream_t st);
// *bad = 1 when a letter code of letters[0, n) is above 24 (0 otherwise).
void launch_check_letters(const uint8_t* letters, uint64_t n, unsigned int* bad, cudaStream_t st);
// out[i] = min(in[i], 24): the codes the score tables see.
void launch_clamp_letters(const uint8_t* in, uint64_t n, uint8_t* out, cudaStream_t st);
// Enumerate seeds of letters [letter_lo, letter_hi) for shapes [0, n_shapes):
// keys[s * (letter_hi - letter_lo) + g - letter_lo] = request << request_shift |
// s << shape_shift | key (shifts from the search's SeedParams), or ~0 when no
// seed.  request (per sequence, optional) tags query seeds with the request
// their target belongs to, so that the join cap counts the query occurrences
// of each request on its own.
void launch_seed_enum(const uint8_t* letters, const uint64_t* offsets, const uint32_t* owner, uint64_t letter_lo,
                      uint64_t letter_hi, int n_shapes, uint64_t* keys, uint32_t* vals, int slot, cudaStream_t st,
                      const uint32_t* request = nullptr);
// The same with 32-bit keys, for a seed key of at most 32 bits and no
// request; "no seed" is 0xFFFFFFFF.  filter (optional, zeroed by the caller):
// each valid key's bit of the query-key bitmap (launch_key_filter's) is set.
void launch_seed_enum(const uint8_t* letters, const uint64_t* offsets, const uint32_t* owner, uint64_t letter_lo,
                      uint64_t letter_hi, int n_shapes, uint32_t* keys, uint32_t* vals, int slot, cudaStream_t st,
                      uint32_t* filter = nullptr, int filter_log2 = 0);
// Bitmap of the query's seed keys for the filtered enumeration: bit
// hash(run_keys[u] & key_mask) of 2^log2_bits is set (filter zeroed first).
void launch_key_filter(const uint64_t* run_keys, uint64_t n, uint64_t key_mask, uint32_t* filter, int log2_bits,
                       cudaStream_t st);
// Reference seeds of letters [letter_lo, letter_hi) whose key's bit is set
// in the filter, appended in no fixed order: counts[0] += kept, counts[1] +=
// valid seeds (kept or not).  keys / vals need room for every seed of the
// range; 32-bit keys for a seed key of at most 32 bits.
void launch_seed_enum_filtered(const uint8_t* letters, const uint64_t* offsets, const uint32_t* owner,
                               uint64_t letter_lo, uint64_t letter_hi, int n_shapes, const uint32_t* filter,
                               int log2_bits, uint64_t* keys, uint32_t* vals, unsigned long long* counts, int slot,
                               cudaStream_t st);
void launch_seed_enum_filtered(const uint8_t* letters, const uint64_t* offsets, const uint32_t* owner,
                               uint64_t letter_lo, uint64_t letter_hi, int n_shapes, const uint32_t* filter,
                               int log2_bits, uint32_t* keys, uint32_t* vals, unsigned long long* counts, int slot,
                               cudaStream_t st);
constexpr uint64_t kNoSeed = ~0ull;
constexpr uint32_t kMaxRequests = 65535;  // request ids of one batch

// A block of the query batch: the targets whose letters lie in [lo, hi).  A
// query key run's entries are in ascending letter order (the key sort is
// stable over the enumeration order), so a block's entries of a run are one
// contiguous sub-range; the join finds it by binary search, tests the
// expansion cap on the count of the whole run (the reference counts a key's
// query occurrences over every target of the run, seed.rs:120-127) and
// expands only the block's entries.
struct JoinBlock {
  const uint32_t* q_vals;      // sorted query entry payloads (letter indices)
  const uint32_t* run_qstart;  // first entry of each run
  uint64_t lo, hi;             // letters of the block
  uint32_t* run_qlo;           // out: first entry of the block in each run
  uint32_t* run_qcount;        // out: entries of the block in each run
};
// For each query run u (unique key, count, start): the reference run [lo, hi)
// with the same key (query key & key_mask) and the number of hits it yields
// under the expansion cap.
// With `first` (launch_bucket_first over the same reference keys), each
// search covers one bucket of keys sharing their bits above `shift`.
// With `blk`, hits count only the block's entries of each run.  With
// d_n_ref, n_ref is *d_n_ref (a count an earlier launch wrote).
void launch_join_count(const uint64_t* run_keys, const uint32_t* run_counts, uint64_t n_runs,
                       const uint64_t* ref_keys, uint64_t n_ref, uint64_t max_expand, uint32_t* run_rlo,
                       uint32_t* run_rcount, uint64_t* run_hits, uint64_t key_mask, cudaStream_t st,
                       const uint32_t* first = nullptr, int shift = 0, const JoinBlock* blk = nullptr,
                       const uint64_t* d_n_ref = nullptr);
void launch_join_count(const uint64_t* run_keys, const uint32_t* run_counts, uint64_t n_runs,
                       const uint32_t* ref_keys, uint64_t n_ref, uint64_t max_expand, uint32_t* run_rlo,
                       uint32_t* run_rcount, uint64_t* run_hits, uint64_t key_mask, cudaStream_t st,
                       const uint32_t* first = nullptr, int shift = 0, const JoinBlock* blk = nullptr,
                       const uint64_t* d_n_ref = nullptr);
// target_hits[t] += hits the join gives target t (runs that pass the cap,
// after launch_join_count without a block): sizes the query blocks.
void launch_target_hits(const uint32_t* run_counts, const uint32_t* run_qstart, const uint32_t* run_rcount,
                        const uint64_t* run_hits, uint64_t n_runs, const uint32_t* q_vals, const uint32_t* q_owner,
                        unsigned long long* target_hits, cudaStream_t st);
// first[b] (b in [0, nb]) = index of the first of n sorted keys whose
// key >> shift is at least b; first[nb] = n.  Keys must be below nb << shift.
// With d_n, n is *d_n (a count an earlier launch wrote).
void launch_bucket_first(const uint64_t* keys, uint64_t n, int shift, uint32_t nb, uint32_t* first, cudaStream_t st,
                         const uint64_t* d_n = nullptr);
void launch_bucket_first(const uint32_t* keys, uint64_t n, int shift, uint32_t nb, uint32_t* first, cudaStream_t st,
                         const uint64_t* d_n = nullptr);

// Layout of the packed 64-bit hit key (target, subject, diag + doff, spos).
// Hit key: target - t_base (tb bits) | subject (sb) | diagonal + doff (db) |
// subject position (pb).  A batch whose full key would pass 64 bits is
// searched in target windows of at most 2^tb targets, t_base the window's
// first target.
struct HitKeyLayout {
  int tb, sb, db, pb;
  int64_t doff;
  uint32_t t_base = 0;
  int total() const { return tb + sb + db + pb; }
};

// Expand every counted run into hits.  Writes hit_keys[h] (packed) when
// keys_mode, otherwise hits[h] = {query seq, qpos, subject seq, spos} taken
// straight from the entries' (seq, pos).
struct JoinExpandArgs {
  const uint64_t* run_hit_off;  // exclusive scan of run_hits, n_runs + 1 entries
  const uint32_t* coarse;       // launch_hit_coarse over run_hit_off (optional)
  int coarse_shift;
  const uint32_t* run_qstart;
  const uint32_t* run_rlo;
  const uint32_t* run_rcount;
  uint64_t n_runs;
  const uint32_t* q_vals;  // query entry payloads
  const uint32_t* r_vals;  // reference entry payloads
  uint64_t n_hits;
  // keys mode: payloads are global letter indices
  const uint32_t* q_owner;      // letter -> target
  const uint64_t* q_offsets;    // target offsets
  const uint32_t* r_owner;      // letter -> subject
  const uint64_t* r_offsets;    // subject offsets
  HitKeyLayout layout;
  uint64_t* hit_keys;
  // entries mode: payloads index seq/pos arrays
  const uint32_t* q_seq;
  const uint32_t* q_pos;
  const uint32_t* r_seq;
  const uint32_t* r_pos;
  uint32_t* hits4;  // 4 x u32 per hit
};
void launch_join_expand(const JoinExpandArgs& a, cudaStream_t st);
// coarse[j] (j in [0, ceil(n_hits >> shift)]) = the run holding hit j << shift
// (the last run for j past the hits): narrows each hit's run search.
void launch_hit_coarse(const uint64_t* run_hit_off, uint64_t n_runs, int shift, uint64_t n_hits, uint32_t* coarse,
                       cudaStream_t st);

// ---- blastx front end (translate.cu) ----------------------------------------
// Per (read, frame) entry i = 6 * read + frame; arrays of 6 * n_reads + 1
// entries, the last one the scans' total.
struct TranslateArgs {
  const uint8_t* nt;            // reads, upper-cased bytes back to back
  const uint64_t* nt_off;       // n_reads + 1
  uint64_t n_reads;
  int64_t min_orf;              // >= 0: for every read; < 0: translate::min_orf_len of each read
  uint8_t* scratch;             // frames before compaction
  const uint64_t* scratch_off;  // exclusive scan of the frame lengths
  uint32_t* keep;               // 1: the frame has a letter below X after masking
  uint64_t* kept_len;           // its length when kept, else 0
  const uint32_t* kept_index;   // exclusive scan of keep: the target index
  const uint64_t* kept_off;     // exclusive scan of kept_len: the target's first letter
  uint8_t* out;                 // kept frames back to back
  uint64_t* out_off;            // n_targets + 1
  uint32_t* out_query;          // read of each target
  uint8_t* out_frame;           // frame 0-5 of each target
};
// len[i] = codons of frame i ((L - offset) / 3), len[6 * n_reads] = 0.
void launch_frame_lengths(const uint64_t* nt_off, uint64_t n_reads, uint64_t* len, cudaStream_t st);
// Translation, ORF masking, keep flags (fills scratch, keep, kept_len).
void launch_translate_frames(const TranslateArgs& a, cudaStream_t st);
// Kept frames into out / out_off / out_query / out_frame.
void launch_compact_frames(const TranslateArgs& a, cudaStream_t st);

// ---- ungapped (ungapped_kernels.cu) -----------------------------------------
// Scores (25x25, int8) in constant memory for X-drop and the band stage.
void upload_score_matrix(const int8_t* scores625, int slot, cudaStream_t st);

struct SegmentOut {  // ungapped.rs:11-17 plus the hit key it came from
  uint32_t q_start, s_start, len;
  int32_t score;
};

// flags[i] = 1 when hit i starts a new (target, subject, diagonal) run.
// flags[i] = 1 where key i >> shift differs from key i - 1 (i < n); with
// d_n, n is *d_n and flags[i] = 0 for i in [*d_n, n).
void launch_run_heads(const uint64_t* keys, uint64_t n, int shift, uint8_t* flags, cudaStream_t st,
                      const int64_t* d_n = nullptr);

struct XdropArgs {
  const uint64_t* hit_keys;
  uint64_t n_hits;
  const uint32_t* run_head_idx;  // compacted indices of run heads
  uint64_t n_runs;
  // when set, n_hits / n_runs are device words written by earlier launches
  // (the host values above then only bound them and size the grid)
  const int64_t* d_n_hits;
  const int64_t* d_n_runs;
  HitKeyLayout layout;
  const uint8_t* q_letters;
  const uint64_t* q_offsets;
  const uint8_t* s_letters;
  const uint64_t* s_offsets;
  int xdrop;
  int cutoff;
  int slot;          // constant bank of the score matrix
  SegmentOut* seg;   // indexed like hits
  uint8_t* keep;     // 1 when hit i produced a kept segment
  unsigned long long* xdrop_count;
};
void launch_xdrop_runs(const XdropArgs& a, cudaStream_t st);

// Plain ungapped::xdrop for explicit anchors (stage entry point).
void launch_xdrop_jobs(const drg_xdrop_job* jobs, uint64_t n, const uint8_t* q_letters, const uint64_t* q_offsets,
                       const uint8_t* s_letters, const uint64_t* s_offsets, int xdrop, drg_segment* out, int slot,
                       cudaStream_t st);

// Band record (search.rs:206-230 + gapped_hsp window, search.rs:303-312).
struct Band {
  uint32_t target, subject;
  int32_t d0, d1;        // diagonal span in window coordinates
  uint32_t q0, n;        // query window [q0, q0 + n)
  int32_t best_score;    // best segment score (band order key)
  uint32_t rank;         // position in the pair's band order
  uint32_t pair;         // pair index
  uint32_t pad;
};

struct BandArgs {
  const uint64_t* seg_keys;  // kept segment keys, sorted
  const SegmentOut* segs;
  uint64_t n_segs;
  const uint32_t* pair_head_idx;  // compacted indices of pair heads (n_pairs + 1, last = n_segs)
  uint64_t n_pairs;
  const int64_t* d_n_pairs;  // when set, the pair count is this device word (n_pairs bounds it)
  HitKeyLayout layout;
  const uint64_t* q_offsets;
  Band* bands;     // indexed like segments
  uint8_t* valid;  // 1 where a band was written
};
void launch_build_bands(const BandArgs& a, cudaStream_t st);

// ---- banded Smith-Waterman, score only (sw_score.cu) -----------------------
struct SwTask {        // one warp: up to 32 bands sharing a query window
  uint32_t first;      // index of the first band in the sorted band order
  uint32_t count;      // 1..32
  uint32_t row_first;  // first DP row of the warp (1-based)
  uint32_t n_strips;   // 16-row strips to run
  uint32_t width;      // widest band of the task, W_max = d1 - d0 + 1
  uint32_t w_min;      // narrowest band of the task
  uint32_t transposed; // 1: rows are the subject, columns the query window (diagonals negated)
  uint32_t pad;
};
// Trace-pass result of one band: where its nibbles are and its first maximum.
struct TraceBand {
  uint64_t trace_off;  // first nibble word of the band
  uint32_t row_first, width;
  int32_t score, best_i, best_j;
  int32_t stride;      // words between consecutive column steps of the band
};
struct SwScoreArgs {
  const Band* bands;
  const uint32_t* order;  // sorted band indices
  const SwTask* tasks;
  uint64_t task_lo, task_hi;  // tasks of this launch
  const uint8_t* q_letters;
  const uint64_t* q_offsets;
  const uint8_t* s_letters;
  const uint64_t* s_offsets;
  int gap_open, gap_extend;
  int32_t* score;     // score mode: per band (indexed like bands)
  int32_t* best_row;  // score mode: first DP row holding the best (0 if none)
  unsigned long long* cells_eval;  // optional: [0] DP cells the lanes evaluated (after skipping), [2] the warps' (idle lanes too)
  uint2* trace;       // trace mode: nibble buffer
  TraceBand* tband;   // trace mode: per band (indexed like bands)
  int8_t scores625[628];  // substitution scores, row-major
};
// One band of the intra-band (one warp per band) kernel.
struct SwBandJob {
  uint32_t band;       // index into bands
  uint32_t row_first;  // first DP row (1-based)
  uint32_t n_strips;   // 16-row strips from row_first
  uint32_t pad;
  uint64_t trace_off;  // trace mode: first uint2 of the band's nibbles
};
struct ExactOut;
// Where a traced band's walk writes (per band t: ops at ops_off[t], n + m
// slots; rev the same bytes as scratch; out[t] the record).
struct WalkEnv {
  const uint2* trace;
  const uint8_t* q_letters;
  const uint64_t* q_offsets;
  const uint8_t* s_letters;
  const uint64_t* s_offsets;
  const uint64_t* ops_off;
  uint8_t* rev;
  uint32_t* ops;
  ExactOut* out;
  int exact_below;  // bands whose best is below this are left to the exact kernel
};
struct SwBandArgs {
  const Band* bands;
  const SwBandJob* jobs;
  uint64_t lo, hi;  // jobs of this launch
  const uint8_t* q_letters;
  const uint64_t* q_offsets;
  const uint8_t* s_letters;
  const uint64_t* s_offsets;
  int gap_open, gap_extend;
  int32_t* score;     // score mode: per band
  int32_t* best_row;  // score mode: first DP row holding the best
  uint2* trace;       // trace mode: nibbles, strip k's step c at trace_off + k (W + 16) + c
  TraceBand* tband;   // trace mode: per band
  WalkEnv walk;       // trace mode: each band is walked right after its DP
  uint32_t xbuf_words;  // set by the launcher
  int8_t scores625[628];
};
size_t sw_band_smem(int max_width);
void launch_sw_band(SwBandArgs a, int max_width, bool trace, cudaStream_t st);
// Bands by width: route 0 (W <= 134), 1 (<= 271), 2 (<= 559) run in groups
// of 8, 16, 32 lanes with rotating strips; route 3 (wider) in the block
// kernel.  The traceback pass's few bands keep a warp each (route 2 up to
// W 559): with several bands per warp too few warps remain to hide the
// step's dependency chain.  max_width matters for route 3 only.
__host__ __device__ inline int sw_band_route(int width, bool trace) {
  if (width > 559) return 3;
  if (trace) return 2;
  return width <= 134 ? 0 : (width <= 271 ? 1 : 2);
}
void launch_sw_band_route(const SwBandArgs& a, int route, int max_width, bool trace, cudaStream_t st);

struct ExactOut;
// Width classes of the packed kernel by the widest band of a warp (the shared
// ring holds W + 1 words per thread); each fits 3 blocks per SM but the last.
constexpr int kSwMinWidth = 17;   // narrower bands use the exact kernel
constexpr int kSwC0 = 136, kSwC1 = 272, kSwC2 = 544, kSwC3 = 1700;
constexpr int kSwClassMax[4] = {kSwC0, kSwC1, kSwC2, kSwC3};  // 4, 2, 1, 1 warps per block
constexpr int kSwMaxWidth = 1700;                       // wider bands use the exact kernel
// The packed kernel's profile bytes hold a score plus the open cost (gap open
// + extend): with larger open costs its bands go to the band kernel.
constexpr int kSwMaxOpenCost = 64;
// Bands whose best can reach this bound are not packed: every H of the packed
// kernel stays below 0x7C00 (its strip maximum folds H on the FMA pipe as
// half-precision bit patterns) and far from the 16-bit limit.
constexpr int kSwPackedMaxBest = 31743;
constexpr int kSwBandMinWidth = kSwC1 + 1;  // score pass: wider bands run one warp per band
constexpr int kSwClasses = 4;
int sw_width_class(int width);  // 0..3, or -1 for the exact kernel
void launch_sw_class(const SwScoreArgs& a, int cls, cudaStream_t st);  // score mode

// ---- device radix sort (radix_sort.cu) --------------------------------------
// The sort's scratch and the epoch of its last pass (look-back words carry
// the epoch of the pass that wrote them).
struct SortScratch {
  DevBuf buf;
  uint32_t epoch = 0;
};
// Where the sorted keys (and values) ended up: the LSD passes alternate between
// the two buffers of each array.
template <typename K>
struct SortResult {
  K* keys;
  uint32_t* vals;
};
// Stable LSD sort of keys[0, n) by bits [begin_bit, end_bit), with optional u32
// values (vals == nullptr: keys only).  n is *d_n when d_n is set (a count
// written by an earlier launch; n_max bounds it and sizes the grids), else
// n_max; n < 2^32.  keys_alt / vals_alt are buffers of the same capacity;
// both buffers of each array are overwritten.  temp is the sort's scratch;
// *d_err becomes non-zero if a tile's bounded wait for an earlier tile gave up
// (the outputs are then not valid).  small_tiles: half the keys per tile.
// No host wait.
template <typename K>
SortResult<K> radix_sort(K* keys, K* keys_alt, uint32_t* vals, uint32_t* vals_alt, uint64_t n_max,
                         const uint64_t* d_n, int begin_bit, int end_bit, SortScratch& temp, uint32_t* d_err,
                         cudaStream_t st, bool small_tiles = false);

// ---- exact DP with traceback (sw_exact.cu) ----------------------------------
struct ExactJob {
  const uint8_t* q;  // query window
  const uint8_t* s;  // subject
  uint32_t n, m;
  int32_t d0, d1;
  uint64_t scratch_off;  // byte offset of this job's scratch (trace + rows)
  uint64_t ops_off;      // index of this job's first op slot (n + m slots)
};
struct ExactOut {
  int32_t score;
  uint32_t q_begin, q_end, s_begin, s_end;
  uint32_t identities, positives, mismatches, gap_openings, gaps, length;
  uint32_t n_ops;
  uint64_t cells;
};
// Sum over x = 0..X of min(x, m) (0 for X < 0).
__host__ __device__ inline uint64_t exact_clamped_sum(int64_t X, uint64_t m) {
  if (X < 0) return 0;
  const uint64_t x = (uint64_t)X;
  if (x <= m) return x * (x + 1) / 2;
  return m * (m + 1) / 2 + (x - m) * m;
}
// Scratch bytes of one exact DP job: the trace bytes of the reference's row
// ranges (gapped.rs:82-97, rows 0..n, columns clamp(i - d1 .. i - d0, 0, m)),
// four int32 rows of the widest row, and in trace mode the reversed op bytes;
// rounded up to 256.  The host sizes the scratch with it and the no-allocation
// entry point lays jobs out on the device with it, so both must agree.
// Lengths below 2^31 and diagonals within +-2^30 keep every term in 64 bits.
__host__ __device__ inline uint64_t exact_scratch_bytes(uint32_t n, uint32_t m, int32_t d0, int32_t d1, bool trace) {
  const int64_t lo_d = d0 < d1 ? d0 : d1, hi_d = d0 < d1 ? d1 : d0;
  int64_t wmax = hi_d - lo_d + 1;
  if (wmax > (int64_t)m + 1) wmax = (int64_t)m + 1;
  uint64_t tb = 0;
  if (trace) {
    // sum over rows i of clamp(i - lo_d, 0, m) - clamp(i - hi_d, 0, m) + 1
    const auto F = [&](int64_t a) { return exact_clamped_sum((int64_t)n - a, m) - exact_clamped_sum(-a - 1, m); };
    tb = (uint64_t)n + 1 + F(lo_d) - F(hi_d);
  }
  uint64_t bytes = ((tb + 15) & ~15ull) + 4ull * 4ull * (uint64_t)wmax;
  if (trace) bytes += (uint64_t)n + (uint64_t)m + 1;  // reversed op bytes
  return (bytes + 255) & ~255ull;
}
// The substitution scores travel with each launch (no shared host state).
void launch_sw_exact_with_matrix(const ExactJob* jobs, uint64_t n_jobs, int gap_open, int gap_extend, bool trace,
                                 uint8_t* scratch, uint32_t* ops, ExactOut* out, const int8_t* scores625,
                                 cudaStream_t st);
// ---- E-value gate (evalue.cu) ---------------------------------------------
struct AlpDev {
  double lambda, k, ln_k, a, b, alpha, beta, sigma, tau, v_thr, c_thr;
};
struct SelectArgs {
  const Band* bands;     // pair-grouped, rank ordered
  const int32_t* score;  // per band
  uint64_t n_bands;
  const uint32_t* pair_first;  // first band of each pair (n_pairs + 1)
  uint64_t n_pairs;
  const uint64_t* q_offsets;
  const uint64_t* s_offsets;
  uint64_t db_letters;
  AlpDev alp;
  double evalue;
  uint32_t max_hsps;
  uint8_t* state;    // per band: 0 skipped, 1 computed-failed, 2 selected, 3 undecided
  uint8_t* verdict;  // per band scratch: the E-value verdict (1 fail, 2 pass, 3 undecided)
  unsigned long long* cells_ref;
  unsigned long long* n_computed;
};
void upload_alp_tables(cudaStream_t st);
void launch_select(const SelectArgs& a, cudaStream_t st);
uint64_t band_cells_host(uint32_t n, uint32_t m, int32_t d0, int32_t d1);

// ---- probe ---------------------------------------------------------------
void run_int_probe(double* lane_ops_per_s, double* mhz, cudaStream_t st);

}  // namespace drg
