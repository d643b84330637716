// CPU ORACLE -- test infrastructure only.
//
// A plain C++ restatement of the diamond-rust protein-search path
// (seed enumeration + complexity mask, double-index join, ungapped X-drop,
// band merge, banded affine Smith-Waterman with traceback, ALP E-values,
// culling, frame merge and outfmt 6).  It exists to check the CUDA product
// and to serve as the timed CPU baseline; nothing in the product links it.
// Every function cites the reference file:line it follows (paths relative to
// the diamond-rust project root).  Parity is pinned against the reference's
// own unit-test vectors and README known answers (tests/test_oracle_*.py).
#pragma once
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>
#include <unordered_map>
#include <optional>
#include <utility>

namespace oracle {

// ---- alphabet.rs ---------------------------------------------------------
constexpr int AA_COUNT = 25;
constexpr int TRUE_AA = 20;
constexpr uint8_t X_LETTER = 23;
constexpr uint8_t STOP_LETTER = 24;
extern const char AA_SYMBOLS[26];
uint8_t encode_byte(uint8_t c);                          // alphabet.rs:54
std::vector<uint8_t> encode(const std::string& raw);     // alphabet.rs:59-68
char decode_byte(uint8_t l);                             // alphabet.rs:71-73
std::string decode(const uint8_t* l, size_t n);          // alphabet.rs:75-77
std::string seq_id(const std::string& header);           // alphabet.rs:92-98

// ---- reduction.rs ---------------------------------------------------------
struct Reduction {
  uint8_t map[AA_COUNT];
  uint64_t size;
  uint8_t bucket(uint8_t letter) const { return map[letter < AA_COUNT ? letter : AA_COUNT - 1]; }
};
Reduction reduction_parse(const std::string& def);       // reduction.rs:19-37
Reduction reduction_murphy10();                          // reduction.rs:48-50
Reduction reduction_diamond9();                          // reduction.rs:52-54
Reduction reduction_none();                              // reduction.rs:65-67
Reduction reduction_for_sensitivity(const std::string&); // reduction.rs:74-80

// ---- shape.rs -------------------------------------------------------------
struct Shape {
  std::string code;
  uint32_t weight = 0, span = 0;
  std::vector<uint32_t> positions;
  // shape.rs:60-75: None when the seed leaves the sequence or holds letter >= 20.
  bool packed(const uint8_t* seq, size_t len, size_t pos, const Reduction& r, uint64_t* key) const;
};
Shape shape_parse(const std::string& code);              // shape.rs:23-44 (throws on bad code)
Shape shape_contiguous(uint32_t weight);                 // shape.rs:47-49
std::vector<Shape> shapes_for(const std::string& sensitivity, size_t limit);  // shape.rs:78-220

// ---- seed.rs --------------------------------------------------------------
struct SeedEntry { uint64_t key; uint32_t seq; uint32_t pos; };
struct SeedHit { uint32_t query, qpos, subject, spos; };
using HitMap = std::unordered_map<uint32_t, std::vector<SeedHit>>;
struct SeqView { const uint8_t* data; size_t len; };

const double* ln_factorial();                            // seed.rs:29-38
bool seed_is_complex(const uint8_t* seq, const Shape& shape, const Reduction& r, double cut);  // seed.rs:46-70
std::vector<SeedEntry> seed_build(const std::vector<SeqView>& seqs, const Shape& shape, const Reduction& r,
                                  uint32_t base, double cut);                                    // seed.rs:76-104
void seed_join_into(const std::vector<SeedEntry>& q, const std::vector<SeedEntry>& r,
                    std::vector<HitMap>& out, size_t max_expand);                                // seed.rs:110-143
std::vector<std::pair<size_t, size_t>> chunks(size_t n, size_t parts);                           // seed.rs:146-164

// ---- matrix.rs / alp.rs -----------------------------------------------------
struct AlpParams {                                       // alp.rs:34-52
  double lambda, k, a, b, alpha, beta, a_j, b_j, alpha_j, beta_j, sigma, tau, vi_thr, vj_thr, c_thr;
  static AlpParams make(double lambda, double k, double alpha, double alpha_v, double sigma, int go, int ge,
                        double u_alpha, double u_alpha_v);                                       // alp.rs:60-92
  double blast_evalue(int raw, size_t qlen, uint64_t db) const;                                  // alp.rs:95-102
  double evalue(int raw, size_t qlen, size_t slen, uint64_t db) const;                           // alp.rs:108-122
  double log_area(double y, double m, double n) const;                                           // alp.rs:125-163
};
double log_erfc(double x);                               // alp.rs:209-237

struct ScoreMatrix {                                     // matrix.rs:22-35
  std::string name;
  int8_t scores[625];
  int gap_open = 0, gap_extend = 0;
  double lambda = 0, k = 0, ln_k = 0;
  bool has_alp = false;
  AlpParams alp{};
  int score(uint8_t a, uint8_t b) const { return scores[(a < 24 ? a : 24) * 25 + (b < 24 ? b : 24)]; }  // matrix.rs:164-168
  int raw_score(double bits) const;                                                              // matrix.rs:182-184
  double bit_score(int raw) const;                                                               // matrix.rs:187-189
  double evalue(int raw, size_t qlen, size_t slen, uint64_t db) const;                           // matrix.rs:195-200
  double evalue_blast(int raw, size_t qlen, uint64_t db) const;                                  // matrix.rs:204-211
};
// matrix.rs:42-98.  Returns false and sets err on unknown matrix / unsupported gaps.
bool score_matrix_standard(const std::string& name, int go, int ge, ScoreMatrix* out, std::string* err);

// ---- ungapped.rs -----------------------------------------------------------
struct Segment {                                         // ungapped.rs:11-33
  size_t q_start, s_start, len;
  int score;
  long diag() const { return (long)q_start - (long)s_start; }
  size_t s_end() const { return s_start + len; }
};
Segment xdrop(const uint8_t* q, size_t qlen, const uint8_t* s, size_t slen, size_t qa, size_t sa,
              const ScoreMatrix& m, int xdrop);          // ungapped.rs:38-88

// ---- hsp.rs / gapped.rs -----------------------------------------------------
enum class Op : uint8_t { Match = 0, Ins = 1, Del = 2 };  // hsp.rs:8-25
struct HspStats {                                        // hsp.rs:29-57
  uint32_t identities = 0, positives = 0, mismatches = 0, gap_openings = 0, gaps = 0, length = 0;
  void add_match(uint8_t a, uint8_t b, const ScoreMatrix& m);
  bool operator==(const HspStats& o) const {
    return identities == o.identities && positives == o.positives && mismatches == o.mismatches &&
           gap_openings == o.gap_openings && gaps == o.gaps && length == o.length;
  }
};
struct Aligned {                                         // gapped.rs:35-43
  int score = 0;
  size_t q_begin = 0, q_end = 0, s_begin = 0, s_end = 0;
  HspStats stats;
  std::vector<std::pair<Op, uint32_t>> ops;
  // Diagnostic only (not in the reference struct): the DP cells evaluated.
  uint64_t cells = 0;
};
size_t band_for(size_t len);                             // gapped.rs:27-32
std::optional<Aligned> extend_span(const uint8_t* q, size_t n, const uint8_t* s, size_t m, long d0, long d1,
                                   const ScoreMatrix& mat, int gap_open, int gap_extend,
                                   uint64_t* cells = nullptr);  // gapped.rs:67-280

struct Hsp {                                             // hsp.rs:65-82
  size_t query = 0, subject = 0;
  uint8_t frame = 0;
  size_t q_begin = 0, q_end = 0, s_begin = 0, s_end = 0;
  int score = 0;
  double bits = 0, evalue = 0;
  HspStats stats;
  std::vector<std::pair<Op, uint32_t>> ops;
  int q_frame() const { return frame < 3 ? frame + 1 : 2 - (int)frame; }
  std::pair<size_t, size_t> nt_range(size_t dna_len) const;
  double pident() const;
  double ppos() const;
  std::string cigar() const;
  std::pair<std::string, std::string> aligned_strings(const uint8_t* q, const uint8_t* s) const;
  std::string btop(const uint8_t* q, const uint8_t* s) const;
};

// ---- db.rs / io.rs ------------------------------------------------------------
struct Record { std::string header, id; std::string raw; };
bool parse_fasta(const std::string& data, std::vector<Record>* out, std::string* err);  // io.rs:40-74
bool read_fasta(const std::string& path, std::vector<Record>* out, std::string* err);   // io.rs:30-38

struct Database {                                        // db.rs:158-291
  std::string path;
  std::vector<uint8_t> data;
  size_t seq_count = 0;
  uint64_t total_letters = 0;
  size_t seq_off_start = 0, def_off_start = 0, letters_start = 0, defs_start = 0;
  bool protein = true;
  size_t len() const { return seq_count; }
  uint64_t seq_offset(size_t i) const;
  uint64_t def_offset(size_t i) const;
  const uint8_t* seq(size_t i) const { return data.data() + letters_start + seq_offset(i); }
  size_t seq_len(size_t i) const { return seq_offset(i + 1) - seq_offset(i); }
  std::string header(size_t i) const;
  std::string id(size_t i) const { return seq_id(header(i)); }
};
bool db_open(const std::string& path, Database* out, std::string* err);                   // db.rs:172-225
bool db_build(const std::string& fasta, const std::string& out_path, std::string* err,
              size_t* n_seqs = nullptr, uint64_t* n_letters = nullptr);                   // db.rs:62-156
std::string with_extension(const std::string& p);                                         // db.rs:40-48

// ---- translate.rs ----------------------------------------------------------------
std::vector<std::vector<uint8_t>> six_frames(const std::string& nt);                        // translate.rs:72-82
std::vector<uint8_t> translate_frame(const std::string& nt, size_t offset);                // translate.rs:54-69
void mask_short_orfs(std::vector<uint8_t>& frame, size_t min_len);                          // translate.rs:101-121
size_t min_orf_len(size_t dna_len, long user);                                              // translate.rs:124-137

// ---- search.rs ------------------------------------------------------------------------
struct SearchConfig {                                    // search.rs:19-80
  ScoreMatrix matrix;
  double evalue = 0.001;
  size_t max_target_seqs = 25, max_hsps = 1;
  std::string sensitivity = "default";
  size_t threads = 1;
  long index_chunks = -1;  // -1 = preset
  double seed_cut = -1;    // < 0 = preset
  bool has_seed_cut = false;
  int ungapped_xdrop() const { return matrix.raw_score(12.3); }
  double seed_cut_for() const;
  size_t index_chunks_for() const;
};
struct Target { size_t query; uint8_t frame; std::vector<uint8_t> letters; };

// Per-run counters of work done (diagnostics, not part of the reference API).
struct RunStats {
  uint64_t query_seeds = 0, ref_seeds = 0, hits = 0, xdrops = 0, segments = 0, bands = 0, dp_cells = 0, hsps = 0;
  double t_seed_join = 0, t_align = 0;
  uint64_t clipped_windows = 0;  // gapped_hsp windows clipped to max_rows (search.rs:303-312)
};

// search.rs:95-146.  Hit maps are built serially, targets aligned on `threads` threads.
std::vector<std::vector<Hsp>> search_run(const Database& db, const std::vector<Target>& targets,
                                         const SearchConfig& cfg, RunStats* stats = nullptr);
// Same, over a plain letters/offsets view (no .dmnd file needed).
struct DbView { const uint8_t* letters; const uint64_t* offsets; size_t n; uint64_t total_letters; };
std::vector<std::vector<Hsp>> search_run_view(const DbView& db, const std::vector<Target>& targets,
                                              const SearchConfig& cfg, RunStats* stats = nullptr);
int cmp_hsp(const Hsp& a, const Hsp& b);                 // search.rs:273-282 (<0: a first)
std::vector<std::vector<Hsp>> merge_frames(std::vector<std::vector<Hsp>> results, const std::vector<Target>& targets,
                                           size_t queries, size_t max_hsps, size_t max_targets);  // search.rs:357-396

// ---- output.rs ------------------------------------------------------------------------
std::string fmt_double(double x);                        // output.rs:235-241
std::string fmt_evalue(double e);                        // output.rs:244-250
// output.rs:116-135: returns field ids (index into kFieldNames) or sets err.
bool parse_outfmt(const std::vector<std::string>& tokens, std::vector<int>* fields, std::string* err);
struct QueryInfo { std::string id, header; const uint8_t* letters; size_t letters_len; size_t dna_len, frame_len; bool translated; };
std::string tabular_row(const Hsp& h, const QueryInfo& q, const Database& db, const std::vector<int>& fields);  // output.rs:150-223

// ---- workflow.rs / cli.rs ---------------------------------------------------------------
int cli_main(int argc, char** argv);                     // main.rs:3-11 + workflow.rs:15-40

}  // namespace oracle
