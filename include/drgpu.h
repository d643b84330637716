/*
 * drgpu -- B200 (sm_100a) protein-search hot path behind a C ABI.
 *
 * The entry points mirror the public functions of the diamond-rust crate on
 * the seed -> join -> ungapped X-drop -> banded Smith-Waterman path, on flat
 * buffers (plain pointers and sizes, no framework types).  Each declaration
 * names the reference function it replaces (file:line in diamond-rust).
 *
 * Conventions
 *  - Every call returns DRG_OK (0) or a DRG_ERR_* code; drg_last_error(ctx)
 *    holds the message (the reference's Error(String), error.rs:11-52).
 *  - Inputs are borrowed for the duration of the call; host pointers unless
 *    the name says "device".
 *  - Outputs allocated by the library are released with drg_free() /
 *    drg_result_free().
 *  - Letters are diamond-rust residue codes 0..24 (alphabet.rs:1-20):
 *    A R N D C Q E G H I L K M F P S T W Y V B J Z X *.
 *  - A context is used by one host thread at a time.
 */
#ifndef DRGPU_H
#define DRGPU_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DRG_OK 0
#define DRG_ERR_INVALID 1   /* bad argument (unknown matrix, shape, preset, size) */
#define DRG_ERR_OOM 2       /* device or host allocation failed */
#define DRG_ERR_CUDA 3      /* CUDA runtime error */
#define DRG_ERR_IO 4        /* file could not be read or written */
#define DRG_ERR_TIMEOUT 5   /* a bounded device-side wait gave up */
#define DRG_ERR_NODEVICE 6  /* no usable CUDA device: there is no CPU fallback */

typedef struct drg_ctx drg_ctx;
typedef struct drg_db drg_db;       /* database resident in device memory */
typedef struct drg_batch drg_batch; /* query batch resident in device memory */

/* seed.rs:14-19 SeedEntry */
typedef struct { uint64_t key; uint32_t seq; uint32_t pos; } drg_seed_entry;
/* seed.rs:21-27 SeedHit */
typedef struct { uint32_t query, qpos, subject, spos; } drg_seed_hit;
/* ungapped.rs:11-17 Segment */
typedef struct { uint64_t q_start, s_start, len; int32_t score; int32_t pad; } drg_segment;
/* ungapped::xdrop arguments: query/subject index into the batch, anchor */
typedef struct { uint32_t query, subject; uint64_t qa, sa; } drg_xdrop_job;
/* gapped::extend_span arguments: query/subject index, diagonal range d0..=d1 */
typedef struct { uint32_t query, subject; int64_t d0, d1; } drg_span_job;
/* gapped.rs:35-43 Aligned (+ hsp.rs:29-57 HspStats); found == 0 is None.
 * ops are run-length encoded as (count << 2 | op), op 0=M 1=I 2=D. */
typedef struct {
  int32_t found, score;
  uint64_t q_begin, q_end, s_begin, s_end;
  uint32_t identities, positives, mismatches, gap_openings, gaps, length;
  uint64_t cells;      /* DP cells of the reference's row ranges */
  uint32_t n_ops, pad; /* ops of this job start at ops_offset */
  uint64_t ops_offset;
} drg_aligned;

/* hsp.rs:65-82 Hsp */
typedef struct {
  uint32_t query, subject;
  uint32_t frame;
  int32_t score;
  uint32_t q_begin, q_end, s_begin, s_end;
  double bits, evalue;
  uint32_t identities, positives, mismatches, gap_openings, gaps, length;
  uint64_t ops_offset;
  uint32_t n_ops, pad;
} drg_hsp;

/* search.rs:19-48 SearchConfig.  Strings are NUL-terminated.
 * index_chunks < 0 and has_seed_cut == 0 keep the preset's values. */
typedef struct {
  const char* matrix;       /* "BLOSUM62" ... ; NULL = BLOSUM62 */
  int32_t gap_open, gap_extend; /* -1 = matrix default */
  double evalue;
  uint32_t max_target_seqs, max_hsps;
  const char* sensitivity;  /* "fast", "default", "sensitive", ... */
  int32_t index_chunks;
  int32_t has_seed_cut;
  double seed_cut;
  uint32_t threads;         /* host threads for the CPU-side steps (0 = all) */
  uint32_t flags;           /* reserved, 0 */
  /* Seed hits held at once before the stages after the join run over them
   * (0 = 2^28).  When one index chunk yields more, the batch's targets are
   * joined in blocks that each stay under it; the expansion cap still counts
   * every target of the batch, so results do not depend on it. */
  uint64_t max_hits_per_pass;
} drg_search_config;

/* Counters and device times of the last search (milliseconds, CUDA events). */
typedef struct {
  uint64_t query_seeds, ref_seeds, hits, unique_hits, xdrops, segments, bands, bands_computed;
  uint64_t dp_cells_ref;    /* cells of the extend_span calls the reference makes */
  uint64_t dp_cells_gpu;    /* cells the score kernel evaluated (incl. padding) */
  uint64_t traced_bands, hsps;
  double ms_total, ms_seed, ms_join, ms_sort, ms_ungapped, ms_bands, ms_sw, ms_select, ms_trace, ms_host;
  double ms_h2d, ms_d2h;
  double ms_sw_kernel;      /* device time of the packed score kernel launches alone */
  uint64_t sw_launches, kernel_launches;
  uint64_t exact_bands;     /* bands the exact kernel handled (not the packed one) */
  /* packed score kernel per class of the widest band in a warp
   * (W <= 136, <= 272, <= 544, <= 1700) */
  uint64_t sw_class_tasks[4];      /* warps (32 bands each at most) */
  uint64_t sw_class_max_steps[4];  /* longest warp: strips x (W + 16) column steps */
  double ms_sw_class[4];           /* device time of each class launch */
  double ms_trace_kernel;          /* device time of the trace-mode kernel launches */
  uint64_t dp_cells_lane;          /* score kernel: each band's own rows x (W + 16), without warp padding */
  uint64_t sw_wide_bands;          /* score pass: bands wider than 272 columns, one warp per band */
  double ms_sw_wide;               /* device time of their launch (concurrent with the classes) */
  uint64_t dp_cells_issued;        /* score kernel: warps x column steps x 16 x 32, idle lanes included */
  uint64_t index_hits;             /* index chunks whose sorted reference seeds came from the db's cache */
  uint64_t sw_transposed_bands;    /* score kernel: bands run with the subject as rows */
  uint64_t seed_shapes;            /* shapes of the preset (seeds per letter enumerated) */
  uint64_t query_blocks;           /* (index chunk, target block) joins: more than the chunks when blocked */
  uint64_t hit_passes;             /* passes of the stages after the join */
} drg_run_stats;

/* search::run result: per-target HSP lists, target_offsets[n_targets+1]. */
typedef struct {
  drg_hsp* hsps;
  uint64_t n_hsps;
  uint64_t* target_offsets;
  uint64_t n_targets;
  uint32_t* ops;
  uint64_t n_ops;
  drg_run_stats stats;
} drg_result;

/* Tile and routing choices of a context (none changes a result).  The
 * defaults are the first value of each list; drg_autotune picks among them.
 *  sw_wide_min_width   score pass: bands at least this wide run in the lane-
 *                      group band kernel instead of one band per lane
 *                      (273; 137 = two bands per warp from 137, 545, 1701 = never)
 *  sw_min_packed_width bands narrower than this run in int32 lanes (exact
 *                      kernel) instead of 16-bit lanes (17, 33)
 *  sw_transpose        short-subject bands may run with the subject as rows (1, 0)
 *  sort_small_tiles    radix sort tiles of 8 (u32) / 6 (u64) keys per thread
 *                      instead of 16 / 12 (0, 1) */
typedef struct {
  int32_t sw_wide_min_width;
  int32_t sw_min_packed_width;
  int32_t sw_transpose;
  int32_t sort_small_tiles;
} drg_tuning;

/* ---- context --------------------------------------------------------- */
/* One context per host thread; up to 8 contexts may be live in a process at
 * a time (each holds its own bank of constant tables, so contexts can search
 * concurrently with different presets).  A ninth returns DRG_ERR_INVALID. */
int drg_ctx_create(int device, drg_ctx** out);
void drg_ctx_destroy(drg_ctx* ctx);
const char* drg_last_error(const drg_ctx* ctx);
const char* drg_version(void);
void drg_free(void* p);

/* The context's tuning (no reference counterpart).  set rejects values
 * outside the lists above with DRG_ERR_INVALID. */
int drg_ctx_get_tuning(const drg_ctx* ctx, drg_tuning* out);
int drg_ctx_set_tuning(drg_ctx* ctx, const drg_tuning* t);

/* ---- stage entry points (seed.rs / ungapped.rs / gapped.rs) ------------ */

/* seed::build (seed.rs:76-104): every seed of every sequence, sorted by key.
 * reduction: 0 = murphy10, 1 = diamond9, 2 = none (reduction.rs:48-67).
 * The order of entries that share a key is unspecified, as in the reference. */
int drg_seed_build(drg_ctx* ctx, const uint8_t* letters, const uint64_t* offsets, uint64_t n_seqs,
                   const char* shape_code, int32_t reduction, uint32_t base, double complexity_cut,
                   drg_seed_entry** out, uint64_t* n_out);

/* seed::join_into (seed.rs:110-143) into n_targets hit maps, returned flat and
 * ordered by (query, subject, qpos - spos, spos); hits are kept with their
 * multiplicity, as the reference pushes them. */
int drg_seed_join(drg_ctx* ctx, const drg_seed_entry* query, uint64_t n_query, const drg_seed_entry* ref,
                  uint64_t n_ref, uint64_t n_targets, uint64_t max_expand, drg_seed_hit** out, uint64_t* n_out);

/* The device radix sort behind seed::build's key sort (seed.rs:102,
 * sort_unstable_by_key) and align_target's hit sort (search.rs:178), from host
 * buffers: keys (key_bytes 4 or 8) and, when vals is not NULL, u32 values are
 * sorted in place by bits [begin_bit, end_bit) of the key, stably (equal keys
 * keep their order).  n < 2^32.  count_on_device = 1 hands the sort its count
 * in device memory, as the search does when a sort follows the kernel that
 * counted its input. */
int drg_radix_sort(drg_ctx* ctx, void* keys, int32_t key_bytes, uint32_t* vals, uint64_t n, int32_t begin_bit,
                   int32_t end_bit, int32_t count_on_device);

/* seed::chunks (seed.rs:146-164): up to `parts` (start, end) pairs. */
int drg_seed_chunks(uint64_t n, uint64_t parts, uint64_t* out_pairs, uint64_t* n_out);

/* ungapped::xdrop (ungapped.rs:38-88) for a batch of anchors. */
int drg_xdrop_batch(drg_ctx* ctx, const uint8_t* q_letters, const uint64_t* q_offsets, uint64_t n_q,
                    const uint8_t* s_letters, const uint64_t* s_offsets, uint64_t n_s, const drg_xdrop_job* jobs,
                    uint64_t n_jobs, const char* matrix, int32_t xdrop, drg_segment* out);

/* gapped::extend_span (gapped.rs:67-280) for a batch of (query, subject, d0, d1).
 * out[n_jobs]; *ops is allocated by the library. */
int drg_extend_span_batch(drg_ctx* ctx, const uint8_t* q_letters, const uint64_t* q_offsets, uint64_t n_q,
                          const uint8_t* s_letters, const uint64_t* s_offsets, uint64_t n_s,
                          const drg_span_job* jobs, uint64_t n_jobs, const char* matrix, int32_t gap_open,
                          int32_t gap_extend, drg_aligned* out, uint32_t** ops, uint64_t* n_ops);

/* gapped::extend_span, score only (gapped.rs:67-203): the band score the
 * search's E-value gate uses, computed by the same packed 16-bit kernel
 * (exact kernel where that one does not apply).  scores[i] = 0 is None. */
int drg_extend_span_scores(drg_ctx* ctx, const uint8_t* q_letters, const uint64_t* q_offsets, uint64_t n_q,
                           const uint8_t* s_letters, const uint64_t* s_offsets, uint64_t n_s,
                           const drg_span_job* jobs, uint64_t n_jobs, const char* matrix, int32_t gap_open,
                           int32_t gap_extend, int32_t* scores, drg_run_stats* stats);

/* gapped::extend_span with traceback, allocating nothing.  This entry point
 * has no counterpart in the reference; it exists for callers that cannot
 * allocate device memory: services whose own pool owns all device memory and
 * forbids library allocations on the request path, and real-time loops that
 * may not take allocator locks.  Results equal drg_extend_span_batch's.
 *  - d_q_letters, d_s_letters: device letters; q_offsets, s_offsets, jobs:
 *    host arrays, copied to the device with cudaMemcpyAsync on `stream`
 *    (pageable arrays may be reused once the call returns; page-locked ones
 *    must stay unchanged until the stream has run the call's work); d_out
 *    (n_jobs entries) and d_ops: device outputs.  Job i's ops start at
 *    d_out[i].ops_offset; d_ops needs sum(n + m) entries.
 *  - Scratch is a static 32 MiB device array per GPU, kept until exit; calls
 *    needing more are rejected with DRG_ERR_INVALID and a message in err.
 *  - Work is queued on `stream` (a cudaStream_t of the current device); all
 *    calls share the scratch array, so calls that overlap on the GPU race.
 *  - The first call on a device sets up the scratch address (with that device
 *    current). */
int drg_extend_span_noalloc(const uint8_t* d_q_letters, const uint64_t* q_offsets, uint64_t n_q,
                            const uint8_t* d_s_letters, const uint64_t* s_offsets, uint64_t n_s,
                            const drg_span_job* jobs, uint64_t n_jobs, const char* matrix, int32_t gap_open,
                            int32_t gap_extend, drg_aligned* d_out, uint32_t* d_ops, uint64_t ops_capacity,
                            void* stream, char* err, size_t err_cap);

/* ---- whole path: search::run (search.rs:95-146) ------------------------ */

/* Database resident in device memory: letters[offsets[i]..offsets[i+1]]. */
int drg_db_create(drg_ctx* ctx, const uint8_t* letters, const uint64_t* offsets, uint64_t n_seqs, drg_db** out);
void drg_db_destroy(drg_db* db);  /* before the db's context is destroyed */

/* Seed index cache of a resident database.  drg_search_batch enumerates and
 * sorts the reference seeds of every index chunk it covers, as the reference
 * does on every run (search.rs:104-126).  With a budget > 0 the sorted seeds of
 * each (shape set, reduction, complexity cut, index chunk) stay in device
 * memory (8 bytes per seed when the seed key fits 32 bits, else 12) for later
 * searches from any context, the least
 * recently used leaving first when the held bytes pass the budget.  Results
 * are the same with or without it.  0 (the default) holds nothing and frees
 * what is held. */
int drg_db_set_index_budget(drg_db* db, uint64_t budget_bytes);
typedef struct {
  uint64_t entries, bytes, hits, misses, evictions;
} drg_index_stats;
int drg_db_index_stats(const drg_db* db, drg_index_stats* out);

/* Query batch (search::Target list, search.rs:82-88) resident in device memory. */
int drg_batch_create(drg_ctx* ctx, const uint8_t* letters, const uint64_t* offsets, const uint32_t* query_index,
                     const uint8_t* frame, uint64_t n_targets, drg_batch** out);
/* A batch holding several independent requests (serving): request[t] is the
 * request of target t (at most 65535).  The seed join's expansion cap counts
 * query occurrences per request (search.rs:109-131 counts them over the whole
 * run), so every request's HSPs equal those of a search of its targets alone;
 * all requests of a batch share the database and the search configuration.
 * A batch whose targets all carry one request id is searched as a plain
 * batch.  No reference counterpart: search::run serves one request per call. */
int drg_batch_create_requests(drg_ctx* ctx, const uint8_t* letters, const uint64_t* offsets,
                              const uint32_t* query_index, const uint8_t* frame, const uint32_t* request,
                              uint64_t n_targets, drg_batch** out);
void drg_batch_destroy(drg_batch* b);

/* blastx front end on the device (translate.rs:54-137 six_frames /
 * mask_short_orfs / min_orf_len, workflow.rs:112-127): the six frames of each
 * read (0-2 forward at offsets 0-2, 3-5 the reverse complement), stop-free
 * stretches shorter than the minimum ORF length masked with X, frames without
 * a letter below X dropped.  nt holds the reads' upper-cased bytes back to
 * back (FASTA records' raw sequence), nt_offsets[n_reads + 1].  min_orf >= 0
 * applies to every read; < 0 uses min_orf_len of each read's length.
 * The kept frames, in (read, frame) order, become a target batch resident in
 * device memory: query index = read, frame = 0-5 (for drg_search_batch, then
 * drg_merge_frames with the read count). */
int drg_batch_create_blastx(drg_ctx* ctx, const uint8_t* nt, const uint64_t* nt_offsets, uint64_t n_reads,
                            int64_t min_orf, drg_batch** out);
/* The same translation, returned to the host: letters, offsets[n_targets + 1],
 * the read and the frame of each target (each freed with drg_free). */
int drg_translate_reads(drg_ctx* ctx, const uint8_t* nt, const uint64_t* nt_offsets, uint64_t n_reads,
                        int64_t min_orf, uint8_t** letters, uint64_t** offsets, uint32_t** query, uint8_t** frame,
                        uint64_t* n_targets);
/* A resident batch's targets: their count, and (when not null, n_targets
 * entries each) the query index and frame of each (drg_merge_frames takes
 * the query indices). */
int drg_batch_targets(const drg_batch* b, uint64_t* n_targets, uint32_t* query, uint8_t* frame);

/* search::run over resident inputs.  Results are per-target HSP lists, each
 * in the reference's order (best target first, search.rs:262-270). */
int drg_search_batch(drg_ctx* ctx, const drg_db* db, const drg_batch* batch, const drg_search_config* cfg,
                     drg_result* out);

/* search::run from host buffers: uploads the database and the targets,
 * searches, downloads the HSPs (the end-to-end drop-in call). */
int drg_search_run(drg_ctx* ctx, const uint8_t* db_letters, const uint64_t* db_offsets, uint64_t n_db,
                   const uint8_t* t_letters, const uint64_t* t_offsets, const uint32_t* t_query,
                   const uint8_t* t_frame, uint64_t n_targets, const drg_search_config* cfg, drg_result* out);

/* search::run from host buffers as the reference orchestrates it
 * (search.rs:95-271), every hot function replaced by its per-stage entry
 * point above: drg_seed_build per shape and chunk, drg_seed_join,
 * drg_xdrop_batch, drg_extend_span_scores, drg_extend_span_batch, with the
 * adjacency rule, band merge, window, E-value walk and culling on the host
 * threads.  Results equal drg_search_run's; it is the plain per-stage drop-in
 * that the fused device pipeline is measured against. */
int drg_search_run_per_stage(drg_ctx* ctx, const uint8_t* db_letters, const uint64_t* db_offsets, uint64_t n_db,
                             const uint8_t* t_letters, const uint64_t* t_offsets, const uint32_t* t_query,
                             const uint8_t* t_frame, uint64_t n_targets, const drg_search_config* cfg,
                             drg_result* out);

/* search::merge_frames (search.rs:357-396) applied to a result, in place:
 * target_offsets becomes per-query offsets (n_queries + 1 entries). */
int drg_merge_frames(drg_result* res, uint64_t n_queries, const uint32_t* t_query, uint64_t max_hsps,
                     uint64_t max_target_seqs);

void drg_result_free(drg_result* res);

/* Autotuner (no reference counterpart): times whole searches of `batch`
 * against `db` under the tuning lists above (coordinate descent from the
 * context's tuning, median of `reps` device-timed searches per candidate,
 * a value kept when 1 % faster) and leaves the best in the context.  With a
 * cache_path, a line "key wide packed transpose small_tiles" per workload
 * kind (device, preset, powers of two of the query and database letters) is
 * read first and appended after a tuning run.  ms_default / ms_best: the
 * median search time under the starting and the chosen tuning (0 when the
 * cache answered).  Results are the same under every tuning. */
int drg_autotune(drg_ctx* ctx, const drg_db* db, const drg_batch* batch, const drg_search_config* cfg,
                 const char* cache_path, int32_t reps, drg_tuning* out, double* ms_default, double* ms_best);

/* ---- statistics (matrix.rs:164-200, alp.rs:108-163) ------------------- */
int drg_matrix_evalue(const char* matrix, int32_t gap_open, int32_t gap_extend, int32_t raw, uint64_t qlen,
                      uint64_t slen, uint64_t db_letters, double* evalue, double* bits);

/* ---- measurement ------------------------------------------------------- */
/* Issue rate of the integer pipe on this device (16x2 DPX max/add-max lane
 * operations per second), measured by a short calibrated kernel. */
int drg_probe_int_peak(drg_ctx* ctx, double* lane_ops_per_s, double* sm_mhz);

#ifdef __cplusplus
}
#endif
#endif /* DRGPU_H */
