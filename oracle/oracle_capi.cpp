// CPU ORACLE -- test infrastructure only (see oracle.h).
// A flat C ABI over the restated reference so Python tests can call each
// stage (ctypes) and compare it with the CUDA product on identical inputs.
#include "oracle.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>

using namespace oracle;

extern "C" {

struct orc_seed_entry { uint64_t key; uint32_t seq, pos; };
struct orc_seed_hit { uint32_t query, qpos, subject, spos; };
struct orc_segment { uint64_t q_start, s_start, len; int32_t score; int32_t pad; };
struct orc_aligned {
  int32_t found, score;
  uint64_t q_begin, q_end, s_begin, s_end;
  uint32_t identities, positives, mismatches, gap_openings, gaps, length;
  uint64_t cells;
  uint32_t n_ops, pad;
};
struct orc_hsp {
  uint32_t query, subject;
  uint32_t frame;
  int32_t score;
  uint32_t q_begin, q_end, s_begin, s_end;
  double bits, evalue;
  uint32_t identities, positives, mismatches, gap_openings, gaps, length;
  uint64_t ops_offset;
  uint32_t n_ops, pad;
};
struct orc_search_config {
  const char* matrix;
  int32_t gap_open, gap_extend;
  double evalue;
  uint32_t max_target_seqs, max_hsps;
  const char* sensitivity;
  int32_t index_chunks;
  int32_t has_seed_cut;
  double seed_cut;
  uint32_t threads;
  uint32_t pad;
};
struct orc_run_stats {
  uint64_t query_seeds, ref_seeds, hits, xdrops, segments, bands, dp_cells, hsps;
  double t_seed_join, t_align;
  uint64_t clipped_windows;
};

static thread_local std::string g_err;
const char* orc_last_error() { return g_err.c_str(); }
void orc_free(void* p) { std::free(p); }

static bool get_matrix(const char* name, int go, int ge, ScoreMatrix* m) {
  return score_matrix_standard(name ? name : "BLOSUM62", go, ge, m, &g_err);
}

static Reduction reduction_by_id(int id) {
  if (id == 1) return reduction_diamond9();
  if (id == 2) return reduction_none();
  return reduction_murphy10();
}

size_t orc_encode(const char* raw, size_t n, uint8_t* out) {
  auto v = encode(std::string(raw, n));
  std::memcpy(out, v.data(), v.size());
  return v.size();
}

double orc_ln_factorial(int n) { return ln_factorial()[n]; }

int orc_seed_is_complex(const uint8_t* seq, const char* shape_code, int reduction, double cut) {
  Shape s = shape_parse(shape_code);
  return seed_is_complex(seq, s, reduction_by_id(reduction), cut) ? 1 : 0;
}

int orc_shape_packed(const uint8_t* seq, size_t len, size_t pos, const char* shape_code, int reduction,
                     uint64_t* key) {
  Shape s = shape_parse(shape_code);
  return s.packed(seq, len, pos, reduction_by_id(reduction), key) ? 1 : 0;
}

// shapes_for(sensitivity, 0) joined with ',' into buf; returns the count.
int orc_shapes_for(const char* sens, char* buf, size_t cap) {
  auto v = shapes_for(sens, 0);
  std::string s;
  for (size_t i = 0; i < v.size(); ++i) s += (i ? "," : "") + v[i].code;
  std::strncpy(buf, s.c_str(), cap);
  return (int)v.size();
}

int orc_seed_build(const uint8_t* letters, const uint64_t* offsets, size_t n_seqs, const char* shape_code,
                   int reduction, uint32_t base, double cut, orc_seed_entry** out, size_t* n_out) {
  try {
    Shape s = shape_parse(shape_code);
    std::vector<SeqView> seqs;
    for (size_t i = 0; i < n_seqs; ++i) seqs.push_back(SeqView{letters + offsets[i], (size_t)(offsets[i + 1] - offsets[i])});
    auto v = seed_build(seqs, s, reduction_by_id(reduction), base, cut);
    *n_out = v.size();
    *out = (orc_seed_entry*)std::malloc(sizeof(orc_seed_entry) * (v.size() + 1));
    for (size_t i = 0; i < v.size(); ++i) (*out)[i] = orc_seed_entry{v[i].key, v[i].seq, v[i].pos};
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

// join_into over n_targets hit maps, flattened in (query, subject, diag, spos) order.
int orc_join(const orc_seed_entry* q, size_t nq, const orc_seed_entry* r, size_t nr, size_t n_targets,
             size_t max_expand, orc_seed_hit** out, size_t* n_out) {
  std::vector<SeedEntry> qv(nq), rv(nr);
  for (size_t i = 0; i < nq; ++i) qv[i] = SeedEntry{q[i].key, q[i].seq, q[i].pos};
  for (size_t i = 0; i < nr; ++i) rv[i] = SeedEntry{r[i].key, r[i].seq, r[i].pos};
  std::vector<HitMap> maps(n_targets);
  seed_join_into(qv, rv, maps, max_expand);
  std::vector<SeedHit> all;
  for (auto& m : maps)
    for (auto& kv : m)
      for (auto& h : kv.second) all.push_back(h);
  std::sort(all.begin(), all.end(), [](const SeedHit& a, const SeedHit& b) {
    if (a.query != b.query) return a.query < b.query;
    if (a.subject != b.subject) return a.subject < b.subject;
    long da = (long)a.qpos - (long)a.spos, db = (long)b.qpos - (long)b.spos;
    if (da != db) return da < db;
    return a.spos < b.spos;
  });
  *n_out = all.size();
  *out = (orc_seed_hit*)std::malloc(sizeof(orc_seed_hit) * (all.size() + 1));
  for (size_t i = 0; i < all.size(); ++i) (*out)[i] = orc_seed_hit{all[i].query, all[i].qpos, all[i].subject, all[i].spos};
  return 0;
}

int orc_chunks(size_t n, size_t parts, uint64_t* out_pairs) {
  auto v = chunks(n, parts);
  for (size_t i = 0; i < v.size(); ++i) {
    out_pairs[2 * i] = v[i].first;
    out_pairs[2 * i + 1] = v[i].second;
  }
  return (int)v.size();
}

int orc_xdrop(const uint8_t* q, size_t qlen, const uint8_t* s, size_t slen, size_t qa, size_t sa,
              const char* matrix, int xd, orc_segment* out) {
  ScoreMatrix m;
  if (!get_matrix(matrix, -1, -1, &m)) return 1;
  Segment g = xdrop(q, qlen, s, slen, qa, sa, m, xd);
  *out = orc_segment{g.q_start, g.s_start, g.len, g.score, 0};
  return 0;
}

// ops written as (count << 2 | op) into ops_out (capacity ops_cap).
int orc_extend_span(const uint8_t* q, size_t n, const uint8_t* s, size_t m, int64_t d0, int64_t d1,
                    const char* matrix, int go, int ge, orc_aligned* out, uint32_t* ops_out, size_t ops_cap) {
  ScoreMatrix mat;
  if (!get_matrix(matrix, go, ge, &mat)) return 1;
  uint64_t cells = 0;
  auto a = extend_span(q, n, s, m, (long)d0, (long)d1, mat, mat.gap_open, mat.gap_extend, &cells);
  std::memset(out, 0, sizeof *out);
  out->cells = cells;
  if (!a) return 0;
  out->found = 1;
  out->score = a->score;
  out->q_begin = a->q_begin;
  out->q_end = a->q_end;
  out->s_begin = a->s_begin;
  out->s_end = a->s_end;
  out->identities = a->stats.identities;
  out->positives = a->stats.positives;
  out->mismatches = a->stats.mismatches;
  out->gap_openings = a->stats.gap_openings;
  out->gaps = a->stats.gaps;
  out->length = a->stats.length;
  out->n_ops = (uint32_t)a->ops.size();
  for (size_t i = 0; i < a->ops.size() && i < ops_cap; ++i)
    ops_out[i] = (a->ops[i].second << 2) | (uint32_t)a->ops[i].first;
  return 0;
}

// ---- small helpers for the reference's unit-test vectors ------------------
size_t orc_decode(const uint8_t* l, size_t n, char* out, size_t cap) {
  std::string s = decode(l, n);
  std::strncpy(out, s.c_str(), cap);
  return s.size();
}
size_t orc_seq_id(const char* header, char* out, size_t cap) {
  std::string s = seq_id(header);
  std::strncpy(out, s.c_str(), cap);
  return s.size();
}
// Reduction bucket of a letter and the reduction's size (id 0 murphy10, 1 diamond9, 2 none).
int orc_bucket(int reduction, uint8_t letter, uint64_t* size) {
  Reduction r = reduction_by_id(reduction);
  if (size) *size = r.size;
  return r.bucket(letter);
}
uint64_t orc_reduction_size_for(const char* sens) { return reduction_for_sensitivity(sens).size; }
double orc_seed_cut_for(const char* sens, int has_cut, double cut) {
  SearchConfig cfg;
  cfg.sensitivity = sens;
  cfg.has_seed_cut = has_cut != 0;
  cfg.seed_cut = cut;
  return cfg.seed_cut_for();
}
size_t orc_index_chunks_for(const char* sens, long chunks) {
  SearchConfig cfg;
  cfg.sensitivity = sens;
  cfg.index_chunks = chunks;
  return cfg.index_chunks_for();
}
size_t orc_translate_frame(const char* nt, size_t offset, uint8_t* out, size_t cap) {
  auto v = translate_frame(nt, offset);
  std::memcpy(out, v.data(), std::min(cap, v.size()));
  return v.size();
}
// Six frames of a nucleotide string, concatenated; lens[6] receives their lengths.
size_t orc_six_frames(const char* nt, uint8_t* out, size_t cap, uint64_t* lens) {
  auto f = six_frames(nt);
  size_t k = 0;
  for (int i = 0; i < 6; ++i) {
    lens[i] = f[i].size();
    for (uint8_t l : f[i])
      if (k < cap) out[k++] = l;
  }
  return k;
}
void orc_mask_short_orfs(uint8_t* frame, size_t n, size_t min_len) {
  std::vector<uint8_t> v(frame, frame + n);
  mask_short_orfs(v, min_len);
  std::memcpy(frame, v.data(), n);
}
size_t orc_min_orf_len(size_t dna_len, long user) { return min_orf_len(dna_len, user); }
// Field ids of an --outfmt token list ("6 qseqid ..." split on spaces), or -1 on error.
int orc_parse_outfmt(const char* tokens, int* fields, int cap) {
  std::vector<std::string> t;
  std::string cur;
  for (const char* p = tokens; *p; ++p) {
    if (*p == ' ') {
      if (!cur.empty()) t.push_back(cur);
      cur.clear();
    } else {
      cur += *p;
    }
  }
  if (!cur.empty()) t.push_back(cur);
  std::vector<int> f;
  if (!parse_outfmt(t, &f, &g_err)) return -1;
  for (int i = 0; i < (int)f.size() && i < cap; ++i) fields[i] = f[i];
  return (int)f.size();
}
int orc_q_frame(uint32_t frame) {
  Hsp h{};
  h.frame = (uint8_t)frame;
  return h.q_frame();
}
void orc_nt_range(uint32_t frame, uint64_t q_begin, uint64_t q_end, uint64_t dna_len, uint64_t* out2) {
  Hsp h{};
  h.frame = (uint8_t)frame;
  h.q_begin = q_begin;
  h.q_end = q_end;
  auto r = h.nt_range(dna_len);
  out2[0] = r.first;
  out2[1] = r.second;
}
double orc_evalue_blast(const char* matrix, int raw, size_t qlen, uint64_t db) {
  ScoreMatrix m;
  if (!get_matrix(matrix, -1, -1, &m)) return -1;
  return m.evalue_blast(raw, qlen, db);
}
int orc_matrix_ok(const char* matrix, int go, int ge) {
  ScoreMatrix m;
  return get_matrix(matrix, go, ge, &m) ? 1 : 0;
}

size_t orc_band_for(size_t len) { return band_for(len); }
double orc_log_erfc(double x) { return log_erfc(x); }

int orc_matrix_info(const char* matrix, int go, int ge, double* lambda_k_lnk, int32_t* gap_oe, int8_t* scores625) {
  ScoreMatrix m;
  if (!get_matrix(matrix, go, ge, &m)) return 1;
  lambda_k_lnk[0] = m.lambda;
  lambda_k_lnk[1] = m.k;
  lambda_k_lnk[2] = m.ln_k;
  gap_oe[0] = m.gap_open;
  gap_oe[1] = m.gap_extend;
  std::memcpy(scores625, m.scores, 625);
  return 0;
}

double orc_evalue(const char* matrix, int go, int ge, int raw, size_t qlen, size_t slen, uint64_t db) {
  ScoreMatrix m;
  if (!get_matrix(matrix, go, ge, &m)) return -1;
  return m.evalue(raw, qlen, slen, db);
}
double orc_bit_score(const char* matrix, int go, int ge, int raw) {
  ScoreMatrix m;
  if (!get_matrix(matrix, go, ge, &m)) return -1;
  return m.bit_score(raw);
}
int orc_raw_score(const char* matrix, int go, int ge, double bits) {
  ScoreMatrix m;
  if (!get_matrix(matrix, go, ge, &m)) return -1;
  return m.raw_score(bits);
}

size_t orc_fmt_evalue(double e, char* buf, size_t cap) {
  std::string s = fmt_evalue(e);
  std::strncpy(buf, s.c_str(), cap);
  return s.size();
}
size_t orc_fmt_double(double x, char* buf, size_t cap) {
  std::string s = fmt_double(x);
  std::strncpy(buf, s.c_str(), cap);
  return s.size();
}

// search::run over a letters/offsets database and a batch of targets.
// Returns per-target HSP lists: target_offsets[n_targets+1] into *hsps, ops in *ops.
int orc_search(const uint8_t* db_letters, const uint64_t* db_offsets, size_t n_db, uint64_t db_total_letters,
               const uint8_t* t_letters, const uint64_t* t_offsets, const uint32_t* t_query, const uint8_t* t_frame,
               size_t n_targets, const orc_search_config* c, int merge, size_t n_queries, orc_hsp** hsps_out,
               uint64_t* target_offsets, uint32_t** ops_out, uint64_t* n_ops_out, orc_run_stats* stats_out) {
  SearchConfig cfg;
  if (!get_matrix(c->matrix, c->gap_open, c->gap_extend, &cfg.matrix)) return 1;
  cfg.evalue = c->evalue;
  cfg.max_target_seqs = c->max_target_seqs;
  cfg.max_hsps = c->max_hsps;
  cfg.sensitivity = c->sensitivity ? c->sensitivity : "default";
  cfg.index_chunks = c->index_chunks;
  cfg.has_seed_cut = c->has_seed_cut != 0;
  cfg.seed_cut = c->seed_cut;
  cfg.threads = c->threads ? c->threads : 1;
  std::vector<Target> targets(n_targets);
  for (size_t i = 0; i < n_targets; ++i) {
    targets[i].query = t_query[i];
    targets[i].frame = t_frame[i];
    targets[i].letters.assign(t_letters + t_offsets[i], t_letters + t_offsets[i + 1]);
  }
  DbView v{db_letters, db_offsets, n_db, db_total_letters};
  RunStats rs;
  auto res = search_run_view(v, targets, cfg, &rs);
  if (merge) res = merge_frames(std::move(res), targets, n_queries, cfg.max_hsps, cfg.max_target_seqs);
  size_t total = 0, total_ops = 0;
  for (auto& r : res) {
    total += r.size();
    for (auto& h : r) total_ops += h.ops.size();
  }
  *hsps_out = (orc_hsp*)std::malloc(sizeof(orc_hsp) * (total + 1));
  *ops_out = (uint32_t*)std::malloc(sizeof(uint32_t) * (total_ops + 1));
  size_t k = 0, ko = 0;
  target_offsets[0] = 0;
  for (size_t t = 0; t < res.size(); ++t) {
    for (auto& h : res[t]) {
      orc_hsp& o = (*hsps_out)[k++];
      o.query = (uint32_t)h.query;
      o.subject = (uint32_t)h.subject;
      o.frame = h.frame;
      o.score = h.score;
      o.q_begin = (uint32_t)h.q_begin;
      o.q_end = (uint32_t)h.q_end;
      o.s_begin = (uint32_t)h.s_begin;
      o.s_end = (uint32_t)h.s_end;
      o.bits = h.bits;
      o.evalue = h.evalue;
      o.identities = h.stats.identities;
      o.positives = h.stats.positives;
      o.mismatches = h.stats.mismatches;
      o.gap_openings = h.stats.gap_openings;
      o.gaps = h.stats.gaps;
      o.length = h.stats.length;
      o.ops_offset = ko;
      o.n_ops = (uint32_t)h.ops.size();
      o.pad = 0;
      for (auto& op : h.ops) (*ops_out)[ko++] = (op.second << 2) | (uint32_t)op.first;
    }
    target_offsets[t + 1] = k;
  }
  *n_ops_out = ko;
  if (stats_out) {
    stats_out->query_seeds = rs.query_seeds;
    stats_out->ref_seeds = rs.ref_seeds;
    stats_out->hits = rs.hits;
    stats_out->xdrops = rs.xdrops;
    stats_out->segments = rs.segments;
    stats_out->bands = rs.bands;
    stats_out->dp_cells = rs.dp_cells;
    stats_out->hsps = rs.hsps;
    stats_out->t_seed_join = rs.t_seed_join;
    stats_out->t_align = rs.t_align;
    stats_out->clipped_windows = rs.clipped_windows;
  }
  return 0;
}

int orc_cli_main(int argc, char** argv) { return cli_main(argc, argv); }

}  // extern "C"
