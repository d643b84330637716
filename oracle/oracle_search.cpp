// CPU ORACLE -- test infrastructure only (see oracle.h).
// search.rs orchestration, db.rs, io.rs, translate.rs, output.rs restated.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <thread>

namespace oracle {

// ---------------------------------------------------------------- search.rs
double SearchConfig::seed_cut_for() const {  // search.rs:55-67
  if (has_seed_cut) return seed_cut;
  const std::string& s = sensitivity;
  if (s == "faster" || s == "fast") return 0.9;
  if (s == "mid-sensitive" || s == "sensitive" || s == "more-sensitive" || s == "very-sensitive" ||
      s == "ultra-sensitive")
    return 1.0;
  return 0.8;
}

size_t SearchConfig::index_chunks_for() const {  // search.rs:69-79
  if (index_chunks >= 0) return std::max<size_t>((size_t)index_chunks, 1);
  if (sensitivity == "very-sensitive" || sensitivity == "ultra-sensitive") return 1;
  return 4;
}

int cmp_hsp(const Hsp& a, const Hsp& b) {  // search.rs:273-282
  if (a.score != b.score) return b.score < a.score ? -1 : 1;
  if (a.evalue < b.evalue) return -1;
  if (a.evalue > b.evalue) return 1;
  if (a.subject != b.subject) return a.subject < b.subject ? -1 : 1;
  return 0;
}

namespace {
struct DbAccess {
  const uint8_t* letters;
  const uint64_t* offsets;
  size_t n;
  uint64_t total;
  const uint8_t* seq(size_t i) const { return letters + offsets[i]; }
  size_t len(size_t i) const { return (size_t)(offsets[i + 1] - offsets[i]); }
};

// search.rs:287-354
std::optional<Hsp> gapped_hsp(const uint8_t* query, size_t qlen, const uint8_t* subject, size_t slen,
                              std::pair<size_t, size_t> anchor, std::pair<long, long> span, size_t band,
                              const SearchConfig& cfg, uint64_t db_letters, const Target& target, uint32_t sid,
                              uint64_t* cells, uint64_t* clipped) {
  size_t row_cells = (size_t)std::max<long>(span.second - span.first, 0) + 1;
  size_t budget = 16000000;
  size_t max_rows = std::max(budget / row_cells, 2 * band + 16);
  size_t q0 = 0, q1 = qlen;
  if (q1 - q0 > max_rows) {
    ++*clipped;  // test counter: windows clipped to max_rows query rows
    q0 = anchor.first >= max_rows / 2 ? anchor.first - max_rows / 2 : 0;
    q1 = std::min(q0 + max_rows, qlen);
    q0 = q1 >= max_rows ? q1 - max_rows : 0;
  }
  size_t s0 = 0, s1 = slen;
  long shift = (long)q0 - (long)s0;
  uint64_t c = 0;
  auto al = extend_span(query + q0, q1 - q0, subject + s0, s1 - s0, span.first - shift, span.second - shift,
                        cfg.matrix, cfg.matrix.gap_open, cfg.matrix.gap_extend, &c);
  *cells += c;
  if (!al) return std::nullopt;
  Hsp h;
  h.query = target.query;
  h.subject = sid;
  h.frame = target.frame;
  h.q_begin = q0 + al->q_begin;
  h.q_end = q0 + al->q_end;
  h.s_begin = s0 + al->s_begin;
  h.s_end = s0 + al->s_end;
  h.score = al->score;
  h.bits = cfg.matrix.bit_score(al->score);
  h.evalue = cfg.matrix.evalue(al->score, qlen, slen, db_letters);
  h.stats = al->stats;
  h.ops = std::move(al->ops);
  return h;
}

struct TargetCounters {
  uint64_t xdrops = 0, segments = 0, bands = 0, cells = 0, hsps = 0, clipped = 0;
};

// search.rs:148-271
std::vector<Hsp> align_target(const DbAccess& db, const Target& target, const HitMap& hits,
                              const SearchConfig& cfg, TargetCounters* tc) {
  std::vector<Hsp> out;
  const uint8_t* query = target.letters.data();
  size_t qlen = target.letters.size();
  if (qlen == 0 || hits.empty()) return out;
  uint64_t db_letters = db.total;
  const ScoreMatrix& matrix = cfg.matrix;
  const int cutoff = 19;
  const int xd = cfg.ungapped_xdrop();
  std::vector<uint32_t> subjects;
  subjects.reserve(hits.size());
  for (auto& kv : hits) subjects.push_back(kv.first);
  std::sort(subjects.begin(), subjects.end());
  std::vector<std::vector<Hsp>> found;
  for (uint32_t sid : subjects) {
    const uint8_t* subject = db.seq(sid);
    size_t slen = db.len(sid);
    if (slen == 0) continue;
    std::vector<SeedHit> seeds = hits.at(sid);
    // sort_unstable_by_key((diag, spos)): equal keys are identical hits.
    std::sort(seeds.begin(), seeds.end(), [](const SeedHit& a, const SeedHit& b) {
      long da = (long)a.qpos - (long)a.spos, dbb = (long)b.qpos - (long)b.spos;
      if (da != dbb) return da < dbb;
      return a.spos < b.spos;
    });
    std::vector<Segment> segments;
    for (const SeedHit& h : seeds) {
      long diag = (long)h.qpos - (long)h.spos;
      if (!segments.empty()) {
        const Segment& last = segments.back();
        if (last.diag() == diag && last.s_end() >= (size_t)h.spos) continue;
      }
      Segment seg = xdrop(query, qlen, subject, slen, h.qpos, h.spos, matrix, xd);
      ++tc->xdrops;
      if (seg.score >= cutoff) segments.push_back(seg);
    }
    if (segments.empty()) continue;
    tc->segments += segments.size();
    // sort_unstable_by_key(Reverse(score)) / (diag) / band order: Rust sorts
    // slices of <= 20 elements with a stable insertion sort, so a stable sort
    // reproduces them exactly there; longer slices with tied keys are
    // unpinned (their order depends on the rustc sort implementation).
    std::stable_sort(segments.begin(), segments.end(),
                     [](const Segment& a, const Segment& b) { return a.score > b.score; });
    size_t band = band_for(qlen);
    std::vector<size_t> order(segments.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return segments[a].diag() < segments[b].diag(); });
    struct Band { long d0, d1; size_t best; };
    std::vector<Band> bands;
    for (size_t idx : order) {
      long diag = segments[idx].diag();
      long b0 = diag - (long)band, b1 = diag + (long)band;
      if (!bands.empty() && b0 <= bands.back().d1) {
        Band& last = bands.back();
        last.d1 = std::max(last.d1, b1);
        if (segments[idx].score > segments[last.best].score) last.best = idx;
      } else {
        bands.push_back(Band{b0, b1, idx});
      }
    }
    std::stable_sort(bands.begin(), bands.end(),
                     [&](const Band& a, const Band& b) { return segments[b.best].score < segments[a.best].score; });
    std::vector<Hsp> hsps;
    for (const Band& bd : bands) {
      if (hsps.size() >= cfg.max_hsps) break;
      ++tc->bands;
      const Segment& seg = segments[bd.best];
      auto hsp = gapped_hsp(query, qlen, subject, slen, {seg.q_start, seg.s_start}, {bd.d0, bd.d1}, band, cfg,
                            db_letters, target, sid, &tc->cells, &tc->clipped);
      if (!hsp) continue;
      if (hsp->evalue <= cfg.evalue) hsps.push_back(std::move(*hsp));
    }
    if (!hsps.empty()) {
      std::stable_sort(hsps.begin(), hsps.end(), [](const Hsp& a, const Hsp& b) { return cmp_hsp(a, b) < 0; });
      found.push_back(std::move(hsps));
    }
  }
  std::stable_sort(found.begin(), found.end(),
                   [](const std::vector<Hsp>& a, const std::vector<Hsp>& b) { return cmp_hsp(a[0], b[0]) < 0; });
  if (found.size() > cfg.max_target_seqs) found.resize(cfg.max_target_seqs);
  for (auto& hs : found) {
    if (hs.size() > cfg.max_hsps) hs.resize(cfg.max_hsps);
    for (auto& h : hs) out.push_back(std::move(h));
  }
  tc->hsps += out.size();
  return out;
}

std::vector<std::vector<Hsp>> run_impl(const DbAccess& db, const std::vector<Target>& targets,
                                       const SearchConfig& cfg, RunStats* stats) {
  std::vector<std::vector<Hsp>> results(targets.size());
  if (targets.empty() || db.n == 0) return results;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<Shape> shapes = shapes_for(cfg.sensitivity, 0);
  Reduction reduction = reduction_for_sensitivity(cfg.sensitivity);
  double seed_cut = cfg.seed_cut_for();
  const double LN_2_CONST = 0.693147180559945309417232121458176568;
  double complexity_cut = seed_cut * LN_2_CONST * (double)shapes[0].weight;
  size_t index_chunks = cfg.index_chunks_for();
  std::vector<SeqView> qseqs;
  for (auto& t : targets) qseqs.push_back(SeqView{t.letters.data(), t.letters.size()});
  std::vector<std::vector<SeedEntry>> query_seeds;
  for (auto& sh : shapes) query_seeds.push_back(seed_build(qseqs, sh, reduction, 0, complexity_cut));
  RunStats local;
  for (auto& qs : query_seeds) local.query_seeds += qs.size();
  std::vector<SeqView> refs;
  for (size_t i = 0; i < db.n; ++i) refs.push_back(SeqView{db.seq(i), db.len(i)});
  std::vector<HitMap> hits(targets.size());
  for (auto [c0, c1] : chunks(db.n, index_chunks)) {
    std::vector<SeqView> part(refs.begin() + c0, refs.begin() + c1);
    for (size_t si = 0; si < shapes.size(); ++si) {
      auto ref_seeds = seed_build(part, shapes[si], reduction, (uint32_t)c0, complexity_cut);
      local.ref_seeds += ref_seeds.size();
      seed_join_into(query_seeds[si], ref_seeds, hits, 4096);
    }
  }
  for (auto& hm : hits)
    for (auto& kv : hm) local.hits += kv.second.size();
  auto t1 = std::chrono::steady_clock::now();
  // rayon par_iter over targets: a pool of cfg.threads workers; results keep target order.
  size_t nthreads = std::max<size_t>(cfg.threads, 1);
  std::atomic<size_t> next{0};
  std::vector<TargetCounters> counters(nthreads);
  auto worker = [&](size_t w) {
    for (;;) {
      size_t ti = next.fetch_add(1);
      if (ti >= targets.size()) break;
      results[ti] = align_target(db, targets[ti], hits[ti], cfg, &counters[w]);
    }
  };
  if (nthreads == 1) {
    worker(0);
  } else {
    std::vector<std::thread> pool;
    for (size_t w = 0; w < nthreads; ++w) pool.emplace_back(worker, w);
    for (auto& th : pool) th.join();
  }
  auto t2 = std::chrono::steady_clock::now();
  for (auto& c : counters) {
    local.xdrops += c.xdrops;
    local.segments += c.segments;
    local.bands += c.bands;
    local.dp_cells += c.cells;
    local.hsps += c.hsps;
    local.clipped_windows += c.clipped;
  }
  local.t_seed_join = std::chrono::duration<double>(t1 - t0).count();
  local.t_align = std::chrono::duration<double>(t2 - t1).count();
  if (stats) *stats = local;
  return results;
}
}  // namespace

std::vector<std::vector<Hsp>> search_run(const Database& db, const std::vector<Target>& targets,
                                         const SearchConfig& cfg, RunStats* stats) {
  std::vector<uint64_t> offs(db.seq_count + 1);
  for (size_t i = 0; i <= db.seq_count; ++i) offs[i] = db.seq_offset(i);
  DbAccess acc{db.data.data() + db.letters_start, offs.data(), db.seq_count, db.total_letters};
  return run_impl(acc, targets, cfg, stats);
}

std::vector<std::vector<Hsp>> search_run_view(const DbView& v, const std::vector<Target>& targets,
                                              const SearchConfig& cfg, RunStats* stats) {
  DbAccess acc{v.letters, v.offsets, v.n, v.total_letters};
  return run_impl(acc, targets, cfg, stats);
}

std::vector<std::vector<Hsp>> merge_frames(std::vector<std::vector<Hsp>> results, const std::vector<Target>& targets,
                                           size_t queries, size_t max_hsps, size_t max_targets) {
  std::vector<std::vector<Hsp>> per_query(queries);
  for (size_t ti = 0; ti < results.size(); ++ti) {
    size_t q = targets[ti].query;
    if (q < queries)
      for (auto& h : results[ti]) per_query[q].push_back(std::move(h));
  }
  for (auto& hsps : per_query) {
    std::stable_sort(hsps.begin(), hsps.end(), [](const Hsp& a, const Hsp& b) { return cmp_hsp(a, b) < 0; });
    std::vector<size_t> order;
    std::unordered_map<size_t, std::vector<Hsp>> by_subject;
    for (auto& h : hsps) {
      auto it = by_subject.find(h.subject);
      if (it != by_subject.end()) {
        if (it->second.size() < max_hsps) it->second.push_back(std::move(h));
      } else if (order.size() < max_targets) {
        order.push_back(h.subject);
        by_subject[h.subject].push_back(std::move(h));
      }
    }
    hsps.clear();
    for (size_t sid : order) {
      auto it = by_subject.find(sid);
      if (it != by_subject.end()) {
        for (auto& h : it->second) hsps.push_back(std::move(h));
        by_subject.erase(it);
      }
    }
  }
  return per_query;
}

// -------------------------------------------------------------------- io.rs
bool parse_fasta(const std::string& data, std::vector<Record>* out, std::string* err) {
  out->clear();
  bool have_header = false, seen_header = false;
  std::string header, seq;
  auto finish = [&]() {
    Record r;
    r.header = header;
    size_t e = 0;
    while (e < header.size() && !(header[e] == ' ' || header[e] == '\t' || header[e] == '\n' || header[e] == '\r' ||
                                  header[e] == 0x0c))
      ++e;
    r.id = header.substr(0, e);
    if (r.id.empty()) r.id = "seq" + std::to_string(std::max<size_t>(seq.size(), 1));
    r.raw = seq;
    seq.clear();
    out->push_back(std::move(r));
  };
  size_t pos = 0;
  while (pos <= data.size()) {
    size_t nl = data.find('\n', pos);
    size_t end = nl == std::string::npos ? data.size() : nl;
    size_t len = end - pos;
    if (len > 0 && data[pos + len - 1] == '\r') --len;
    const char* line = data.data() + pos;
    if (len > 0 && line[0] == '>') {
      if (have_header) finish();
      seen_header = true;
      std::string text(line + 1, len - 1);
      size_t b = 0, e = text.size();
      auto ws = [](char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == 0x0b || c == 0x0c; };
      while (b < e && ws(text[b])) ++b;
      while (e > b && ws(text[e - 1])) --e;
      header = text.substr(b, e - b);
      have_header = true;
    } else if (have_header) {
      for (size_t k = 0; k < len; ++k) {
        unsigned char c = (unsigned char)line[k];
        if (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == 0x0c || c == '-' || c == '.') continue;
        seq.push_back((char)toupper(c));
      }
    } else if (len > 0 && line[0] != ';' && line[0] != '#') {
      *err = "malformed FASTA: sequence data found before the first '>' header";
      return false;
    }
    if (nl == std::string::npos) break;
    pos = nl + 1;
  }
  if (have_header) finish();
  if (!seen_header && !data.empty()) {
    *err = "malformed FASTA: no '>' header found";
    return false;
  }
  return true;
}

static bool read_file(const std::string& path, std::string* out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  std::ostringstream ss;
  ss << f.rdbuf();
  *out = ss.str();
  return true;
}

bool read_fasta(const std::string& path, std::vector<Record>* out, std::string* err) {
  std::string data;
  if (!read_file(path, &data)) {
    *err = "cannot read " + path;
    return false;
  }
  if (!parse_fasta(data, out, err)) return false;
  if (out->empty()) {
    *err = path + ": no FASTA records found";
    return false;
  }
  return true;
}

// -------------------------------------------------------------------- db.rs
static const char MAGIC[9] = "DRDMND01";
static const size_t HEADER_LEN = 72;
static uint64_t rd64(const uint8_t* p) {
  uint64_t v;
  std::memcpy(&v, p, 8);
  return v;
}
uint64_t Database::seq_offset(size_t i) const { return rd64(data.data() + seq_off_start + 8 * i); }
uint64_t Database::def_offset(size_t i) const { return rd64(data.data() + def_off_start + 8 * i); }
std::string Database::header(size_t i) const {
  size_t lo = defs_start + def_offset(i), hi = defs_start + def_offset(i + 1);
  return std::string((const char*)data.data() + lo, hi - lo);
}

std::string with_extension(const std::string& p) {
  size_t slash = p.find_last_of('/');
  std::string base = slash == std::string::npos ? p : p.substr(slash + 1);
  size_t dot = base.find_last_of('.');
  if (dot != std::string::npos && dot > 0) return p;  // Path::extension is Some
  return p + ".dmnd";
}

bool db_open(const std::string& path0, Database* out, std::string* err) {
  std::string path = path0;
  {
    std::ifstream f(path);
    if (!f) {
      std::string alt = with_extension(path);
      std::ifstream g(alt);
      if (!g) {
        *err = "Database file not found: " + path0;
        return false;
      }
      path = alt;
    }
  }
  std::string raw;
  if (!read_file(path, &raw)) {
    *err = "cannot read " + path;
    return false;
  }
  Database db;
  db.path = path;
  db.data.assign(raw.begin(), raw.end());
  if (db.data.size() < HEADER_LEN) {
    *err = path + ": not a diamond-rust database (file too short)";
    return false;
  }
  if (std::memcmp(db.data.data(), MAGIC, 8) != 0) {
    *err = path + ": not a diamond-rust database (bad magic). Build one with `diamond-rust makedb`.";
    return false;
  }
  uint32_t version, flags;
  std::memcpy(&version, db.data.data() + 8, 4);
  std::memcpy(&flags, db.data.data() + 12, 4);
  if (version != 1) {
    *err = path + ": database version " + std::to_string(version) + " is not supported (expected 1)";
    return false;
  }
  const uint8_t* d = db.data.data();
  db.seq_count = (size_t)rd64(d + 16);
  db.total_letters = rd64(d + 24);
  uint64_t defs_len = rd64(d + 32);
  db.seq_off_start = (size_t)rd64(d + 40);
  db.def_off_start = (size_t)rd64(d + 48);
  db.letters_start = (size_t)rd64(d + 56);
  db.defs_start = (size_t)rd64(d + 64);
  if (db.defs_start + defs_len != db.data.size()) {
    *err = path + ": truncated or corrupt database";
    return false;
  }
  if (db.seq_off_start + 8 * (db.seq_count + 1) > db.data.size() ||
      db.def_off_start + 8 * (db.seq_count + 1) > db.data.size()) {
    *err = path + ": corrupt offset table";
    return false;
  }
  db.protein = (flags & 1) != 0;
  *out = std::move(db);
  return true;
}

bool db_build(const std::string& fasta, const std::string& out_path, std::string* err, size_t* n_seqs,
              uint64_t* n_letters) {
  std::vector<Record> recs;
  if (!read_fasta(fasta, &recs, err)) return false;
  size_t n = recs.size();
  std::vector<std::vector<uint8_t>> enc(n);
  for (size_t i = 0; i < n; ++i) enc[i] = encode(recs[i].raw);
  std::vector<uint64_t> so, dof;
  uint64_t letters = 0, defs = 0;
  for (size_t i = 0; i < n; ++i) {
    so.push_back(letters);
    letters += enc[i].size();
    dof.push_back(defs);
    defs += recs[i].header.size();
  }
  so.push_back(letters);
  dof.push_back(defs);
  uint64_t seq_off_start = HEADER_LEN, def_off_start = seq_off_start + 8 * (n + 1),
           letters_start = def_off_start + 8 * (n + 1), defs_start = letters_start + letters;
  std::ofstream f(out_path, std::ios::binary);
  if (!f) {
    *err = "cannot create " + out_path;
    return false;
  }
  uint32_t version = 1, flags = 1;
  uint64_t nn = n;
  f.write(MAGIC, 8);
  f.write((const char*)&version, 4);
  f.write((const char*)&flags, 4);
  for (uint64_t v : {nn, letters, defs, seq_off_start, def_off_start, letters_start, defs_start})
    f.write((const char*)&v, 8);
  for (uint64_t v : so) f.write((const char*)&v, 8);
  for (uint64_t v : dof) f.write((const char*)&v, 8);
  for (auto& e : enc) f.write((const char*)e.data(), (std::streamsize)e.size());
  for (auto& r : recs) f.write(r.header.data(), (std::streamsize)r.header.size());
  if (n_seqs) *n_seqs = n;
  if (n_letters) *n_letters = letters;
  return true;
}

// -------------------------------------------------------------- translate.rs
static const char CODON[65] = "FFLLSSSSYY**CC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG";
static uint8_t nt_base(char b) {
  switch (b) {
    case 'T': case 't': case 'U': case 'u': return 0;
    case 'C': case 'c': return 1;
    case 'A': case 'a': return 2;
    case 'G': case 'g': return 3;
    default: return 4;
  }
}
static char complement(char b) {
  switch (b) {
    case 'A': return 'T'; case 'T': return 'A'; case 'C': return 'G'; case 'G': return 'C';
    case 'U': return 'A'; case 'R': return 'Y'; case 'Y': return 'R'; case 'S': return 'S';
    case 'W': return 'W'; case 'K': return 'M'; case 'M': return 'K'; case 'B': return 'V';
    case 'V': return 'B'; case 'D': return 'H'; case 'H': return 'D'; case 'N': return 'N';
    default: return b;
  }
}
std::vector<uint8_t> translate_frame(const std::string& nt, size_t offset) {
  std::vector<uint8_t> out;
  for (size_t i = offset; i + 3 <= nt.size(); i += 3) {
    uint8_t a = nt_base(nt[i]), b = nt_base(nt[i + 1]), c = nt_base(nt[i + 2]);
    if (a > 3 || b > 3 || c > 3) out.push_back(X_LETTER);
    else out.push_back(encode_byte((uint8_t)CODON[a * 16 + b * 4 + c]));
  }
  return out;
}
std::vector<std::vector<uint8_t>> six_frames(const std::string& nt) {
  std::string rc(nt.rbegin(), nt.rend());
  for (auto& c : rc) c = complement(c);
  std::vector<std::vector<uint8_t>> frames;
  for (size_t o = 0; o < 3; ++o) frames.push_back(translate_frame(nt, o));
  for (size_t o = 0; o < 3; ++o) frames.push_back(translate_frame(rc, o));
  return frames;
}
void mask_short_orfs(std::vector<uint8_t>& frame, size_t min_len) {
  if (min_len <= 1) return;
  size_t begin = 0;
  for (size_t i = 0; i < frame.size(); ++i) {
    if (frame[i] == STOP_LETTER) {
      if (i - begin < min_len)
        for (size_t k = begin; k < i; ++k) frame[k] = X_LETTER;
      begin = i + 1;
    }
  }
  if (frame.size() - begin < min_len)
    for (size_t k = begin; k < frame.size(); ++k) frame[k] = X_LETTER;
}
size_t min_orf_len(size_t dna_len, long user) {
  if (user >= 0) return (size_t)user;
  return dna_len < 30 ? 1 : (dna_len < 100 ? 20 : 40);
}

// ----------------------------------------------------------------- output.rs
static const char* kFieldNames[] = {"qseqid", "qlen", "sseqid", "slen", "qstart", "qend", "sstart", "send",
                                    "qseq", "sseq", "evalue", "bitscore", "score", "length", "pident",
                                    "nident", "mismatch", "positive", "gapopen", "gaps", "ppos", "qframe",
                                    "qcovhsp", "scovhsp", "cigar", "btop", "qtitle", "stitle", "full_sseq",
                                    "qseq_translated", "qstrand"};
enum { F_QSEQID, F_QLEN, F_SSEQID, F_SLEN, F_QSTART, F_QEND, F_SSTART, F_SEND, F_QSEQ, F_SSEQ, F_EVALUE,
       F_BITSCORE, F_SCORE, F_LENGTH, F_PIDENT, F_NIDENT, F_MISMATCH, F_POSITIVE, F_GAPOPEN, F_GAPS, F_PPOS,
       F_QFRAME, F_QCOVHSP, F_SCOVHSP, F_CIGAR, F_BTOP, F_QTITLE, F_STITLE, F_FULL_SSEQ, F_QSEQ_TRANSLATED,
       F_QSTRAND, F_COUNT };

std::string fmt_double(double x) {
  char buf[64];
  if (x >= 100.0) {
    snprintf(buf, sizeof buf, "%lld", (long long)std::floor(x));
  } else {
    snprintf(buf, sizeof buf, "%.1f", x);
  }
  return buf;
}

std::string fmt_evalue(double e) {
  if (!std::isfinite(e) || e <= 0.0) return "0.0";
  char buf[64];
  snprintf(buf, sizeof buf, "%.2e", e);  // d.dde[+-]XX -> Rust's d.dde[-]X
  std::string s(buf);
  size_t p = s.find('e');
  std::string mant = s.substr(0, p);
  int ex = std::atoi(s.c_str() + p + 1);
  return mant + "e" + std::to_string(ex);
}

bool parse_outfmt(const std::vector<std::string>& tokens, std::vector<int>* fields, std::string* err) {
  fields->clear();
  static const int defaults[] = {F_QSEQID, F_SSEQID, F_PIDENT, F_LENGTH, F_MISMATCH, F_GAPOPEN,
                                 F_QSTART, F_QEND,   F_SSTART, F_SEND,   F_EVALUE,   F_BITSCORE};
  if (tokens.empty()) {
    fields->assign(std::begin(defaults), std::end(defaults));
    return true;
  }
  const std::string& first = tokens[0];
  if (first != "6") {
    if (first == "0" || first == "5" || first == "102") *err = "--outfmt " + first + " is not supported, use 6 (tabular)";
    else *err = "invalid --outfmt value \"" + first + "\"";
    return false;
  }
  if (tokens.size() <= 1) {
    fields->assign(std::begin(defaults), std::end(defaults));
    return true;
  }
  for (size_t i = 1; i < tokens.size(); ++i) {
    int f = -1;
    for (int k = 0; k < F_COUNT; ++k)
      if (tokens[i] == kFieldNames[k]) f = k;
    if (f < 0) {
      *err = "Invalid output field: " + tokens[i];
      return false;
    }
    fields->push_back(f);
  }
  return true;
}

std::string tabular_row(const Hsp& h, const QueryInfo& q, const Database& db, const std::vector<int>& fields) {
  const uint8_t* subject = db.seq(h.subject);
  size_t subject_len = db.seq_len(h.subject);
  size_t qb = h.q_begin, qe = h.q_end;
  if (q.translated) {
    auto r = h.nt_range(q.dna_len);
    qb = r.first;
    qe = r.second;
  }
  size_t query_len = q.translated ? q.dna_len : q.frame_len;
  std::string row;
  for (size_t fi = 0; fi < fields.size(); ++fi) {
    std::string v;
    switch (fields[fi]) {
      case F_QSEQID: v = q.id; break;
      case F_QLEN: v = std::to_string(query_len); break;
      case F_SSEQID: v = db.id(h.subject); break;
      case F_SLEN: v = std::to_string(subject_len); break;
      case F_QSTART: v = std::to_string(qb + 1); break;
      case F_QEND: v = std::to_string(qe); break;
      case F_SSTART: v = std::to_string(h.s_begin + 1); break;
      case F_SEND: v = std::to_string(h.s_end); break;
      case F_QSEQ: v = h.aligned_strings(q.letters, subject).first; break;
      case F_SSEQ: v = h.aligned_strings(q.letters, subject).second; break;
      case F_EVALUE: v = fmt_evalue(h.evalue); break;
      case F_BITSCORE: v = fmt_double(h.bits); break;
      case F_SCORE: v = std::to_string(h.score); break;
      case F_LENGTH: v = std::to_string(h.stats.length); break;
      case F_PIDENT: v = fmt_double(h.pident()); break;
      case F_NIDENT: v = std::to_string(h.stats.identities); break;
      case F_MISMATCH: v = std::to_string(h.stats.mismatches); break;
      case F_POSITIVE: v = std::to_string(h.stats.positives); break;
      case F_GAPOPEN: v = std::to_string(h.stats.gap_openings); break;
      case F_GAPS: v = std::to_string(h.stats.gaps); break;
      case F_PPOS: v = fmt_double(h.ppos()); break;
      case F_QFRAME: v = std::to_string(h.q_frame()); break;
      case F_QCOVHSP:
        v = query_len == 0 ? "0.0" : fmt_double((double)(qe - qb) * 100.0 / (double)query_len);
        break;
      case F_SCOVHSP:
        v = subject_len == 0 ? "0.0" : fmt_double((double)(h.s_end - h.s_begin) * 100.0 / (double)subject_len);
        break;
      case F_CIGAR: v = h.cigar(); break;
      case F_BTOP: v = h.btop(q.letters, subject); break;
      case F_QTITLE: v = q.header; break;
      case F_STITLE: v = db.header(h.subject); break;
      case F_FULL_SSEQ: v = decode(subject, subject_len); break;
      case F_QSEQ_TRANSLATED: {
        size_t end = std::min(h.q_end, q.letters_len);
        size_t begin = std::min(h.q_begin, end);
        v = decode(q.letters + begin, end - begin);
        break;
      }
      case F_QSTRAND: v = h.frame >= 3 ? "-" : "+"; break;
    }
    if (fi) row += '\t';
    row += v;
  }
  row += '\n';
  return row;
}

}  // namespace oracle
