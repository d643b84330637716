// CPU ORACLE -- test infrastructure only (see oracle.h).
// Alphabet, reductions, shapes, seeds, X-drop, banded SW, HSP rendering,
// score matrices and ALP statistics, restated from the reference.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace oracle {

#include "score_tables.inc"

// ---------------------------------------------------------------- alphabet.rs
const char AA_SYMBOLS[26] = "ARNDCQEGHILKMFPSTWYVBJZX*";

namespace {
struct EncodeTable {
  uint8_t t[256];
  EncodeTable() {  // alphabet.rs:24-44
    for (int i = 0; i < 256; ++i) t[i] = X_LETTER;
    for (int i = 0; i < 25; ++i) {
      uint8_t c = (uint8_t)AA_SYMBOLS[i];
      t[c] = (uint8_t)i;
      if (c >= 'A' && c <= 'Z') t[c - 'A' + 'a'] = (uint8_t)i;
    }
    t['U'] = 4; t['u'] = 4; t['O'] = 11; t['o'] = 11;
  }
};
const EncodeTable kEnc;
bool ascii_ws(uint8_t c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == 0x0c; }
}  // namespace

uint8_t encode_byte(uint8_t c) { return kEnc.t[c]; }

std::vector<uint8_t> encode(const std::string& raw) {
  std::vector<uint8_t> out;
  out.reserve(raw.size());
  for (unsigned char c : raw) {
    if (ascii_ws(c) || c == '-' || c == '.') continue;
    out.push_back(kEnc.t[c]);
  }
  return out;
}

char decode_byte(uint8_t l) { return AA_SYMBOLS[l < AA_COUNT ? l : AA_COUNT - 1]; }

std::string decode(const uint8_t* l, size_t n) {
  std::string s(n, ' ');
  for (size_t i = 0; i < n; ++i) s[i] = decode_byte(l[i]);
  return s;
}

std::string seq_id(const std::string& header) {  // alphabet.rs:92-98
  size_t b = 0;
  while (b < header.size() && (header[b] == '>' || header[b] == ' ')) ++b;
  size_t e = b;
  while (e < header.size() && !ascii_ws((uint8_t)header[e])) ++e;
  return header.substr(b, e - b);
}

// --------------------------------------------------------------- reduction.rs
Reduction reduction_parse(const std::string& def) {
  Reduction r;
  for (int i = 0; i < AA_COUNT; ++i) r.map[i] = 0xff;
  uint8_t bucket = 0;
  size_t i = 0;
  while (i < def.size()) {
    while (i < def.size() && ascii_ws((uint8_t)def[i])) ++i;
    if (i >= def.size()) break;
    while (i < def.size() && !ascii_ws((uint8_t)def[i])) {
      uint8_t l = encode_byte((uint8_t)def[i]);
      if (l < TRUE_AA) r.map[l] = bucket;
      ++i;
    }
    ++bucket;
  }
  if (bucket == 0) throw std::runtime_error("empty reduction definition");
  r.size = bucket;
  return r;
}
Reduction reduction_murphy10() { return reduction_parse("A KR EDNQ C G H ILVM FYW P ST"); }
Reduction reduction_diamond9() { return reduction_parse("A G P CH ST NDE RQK FWY ILMV"); }
Reduction reduction_none() { return reduction_parse("A R N D C Q E G H I L K M F P S T W Y V"); }
Reduction reduction_for_sensitivity(const std::string& s) {
  return s == "very-sensitive" ? reduction_diamond9() : reduction_murphy10();
}

// ------------------------------------------------------------------- shape.rs
Shape shape_parse(const std::string& code) {
  Shape s;
  s.code = code;
  for (size_t i = 0; i < code.size(); ++i) {
    if (code[i] == '1') {
      s.positions.push_back((uint32_t)i);
      s.span = (uint32_t)i + 1;
    } else if (code[i] == '0') {
      s.span = (uint32_t)i + 1;
    } else {
      throw std::invalid_argument("invalid seed shape " + code + ": expected only 0/1");
    }
  }
  if (s.positions.empty()) throw std::invalid_argument("seed shape " + code + " has weight 0");
  s.weight = (uint32_t)s.positions.size();
  return s;
}

Shape shape_contiguous(uint32_t w) { return shape_parse(std::string(w, '1')); }

bool Shape::packed(const uint8_t* seq, size_t len, size_t pos, const Reduction& r, uint64_t* key) const {
  if (pos + span > len) return false;
  uint64_t k = 0;
  for (uint32_t off : positions) {
    uint8_t l = seq[pos + off];
    if (l >= 20) return false;
    k = k * r.size + r.bucket(l);
  }
  *key = k;
  return true;
}

std::vector<Shape> shapes_for(const std::string& sens, size_t limit) {
  static const std::vector<std::string> fast = {"1101110101101111"};
  static const std::vector<std::string> deflt = {"111101110111", "111011010010111"};
  static const std::vector<std::string> mid = {"11110110111",    "1101100111101",    "1110010101111",
                                               "11010101100111", "11101110001011",   "1110100100010111",
                                               "1101000011010111", "1110011000011011"};
  static const std::vector<std::string> sens16 = {
      "1011110111",     "110100100010111",  "11001011111",      "101110001111",
      "11011101100001", "1111010010101",    "111001001001011",  "10101001101011",
      "111101010011",   "1111000010000111", "1100011011011",    "1101010000011011",
      "1110001010101001", "110011000110011", "11011010001101",  "1101001100010011"};
  static const std::vector<std::string> very = {
      "11110111",          "11100100111",        "110010101011",        "11010001001011",
      "10101100001101",    "110100100100011",    "1010010100010011",    "1100101000001011",
      "11100000100010101", "11000100010010011",  "11010000001000111",   "110001001000010011",
      "1010001000100001011", "1100010100000010011", "1100100000101000011", "1101000010000001011"};
  static const std::vector<std::string> ultra = {
      "1111111",          "11101111",         "110011111",        "110110111",        "111111001",
      "1010111011",       "1011110101",       "1111000111",       "10011110011",      "10101101101",
      "10111010101",      "11001010111",      "11001100111",      "11010101101",      "11110001011",
      "100111010011",     "101100110101",     "101110000111",     "110100101011",     "110110001101",
      "111000110011",     "1010001011011",    "1010101000111",    "1010110100011",    "1100100110011",
      "1100101001011",    "1101001100101",    "1101010101001",    "1110001010101",    "1110010010011",
      "10100001101101",   "11000100010111",   "11010000100111",   "11010100110001",   "11101000011001",
      "11110000001101",   "11110100000011",   "101001000001111",  "110000100101011",  "110010010000111",
      "110101100001001",  "110110000010011",  "111001000100011",  "111100000100101",  "1000110010010101",
      "1001000100101101", "1001000110011001", "1010001001001011", "1010001010010011", "1010010001010101",
      "1010010100010011", "1010010101001001", "1010100000101011", "1010100011000101", "1011000010001011",
      "1100010000111001", "1100010010001011", "1100100001001011", "1100100100100011", "1100110000001101",
      "1101000100010011", "1101000110000101", "1110000001010011", "1110100000010101"};
  const std::vector<std::string>* codes = &deflt;
  if (sens == "faster" || sens == "fast") codes = &fast;
  else if (sens == "default") codes = &deflt;
  else if (sens == "mid-sensitive") codes = &mid;
  else if (sens == "sensitive" || sens == "more-sensitive") codes = &sens16;
  else if (sens == "very-sensitive") codes = &very;
  else if (sens == "ultra-sensitive") codes = &ultra;
  size_t n = limit == 0 ? codes->size() : std::min(limit, codes->size());
  std::vector<Shape> out;
  for (size_t i = 0; i < n; ++i) out.push_back(shape_parse((*codes)[i]));
  return out;
}

// -------------------------------------------------------------------- seed.rs
const double* ln_factorial() {
  static double t[33];
  static bool init = [] {
    t[0] = 0.0;
    t[1] = 0.0;
    for (int n = 2; n < 33; ++n) t[n] = t[n - 1] + std::log((double)n);
    return true;
  }();
  (void)init;
  return t;
}

bool seed_is_complex(const uint8_t* seq, const Shape& shape, const Reduction& r, double cut) {
  if (cut <= 0.0) return true;
  uint32_t count[32] = {0};
  for (uint32_t off : shape.positions) {
    uint8_t letter = seq[off];
    if (letter >= 20) return false;
    size_t b = r.bucket(letter);
    if (b >= 32) return false;
    count[b] += 1;
  }
  const double* lnf = ln_factorial();
  double entropy = lnf[shape.weight];
  for (int b = 0; b < 32; ++b)
    if (count[b] > 0) entropy -= lnf[count[b]];
  return entropy >= cut;
}

std::vector<SeedEntry> seed_build(const std::vector<SeqView>& seqs, const Shape& shape, const Reduction& r,
                                  uint32_t base, double cut) {
  std::vector<SeedEntry> out;
  for (size_t i = 0; i < seqs.size(); ++i) {
    const SeqView& s = seqs[i];
    if (s.len < shape.span) continue;
    for (size_t pos = 0; pos + shape.span <= s.len; ++pos) {
      uint64_t key;
      if (!shape.packed(s.data, s.len, pos, r, &key)) continue;
      if (!seed_is_complex(s.data + pos, shape, r, cut)) continue;
      out.push_back(SeedEntry{key, base + (uint32_t)i, (uint32_t)pos});
    }
  }
  // sort_unstable_by_key(key): the order inside one key is unspecified; a full
  // (key, seq, pos) order is one valid instance and keeps the oracle deterministic.
  std::sort(out.begin(), out.end(), [](const SeedEntry& a, const SeedEntry& b) {
    if (a.key != b.key) return a.key < b.key;
    if (a.seq != b.seq) return a.seq < b.seq;
    return a.pos < b.pos;
  });
  return out;
}

void seed_join_into(const std::vector<SeedEntry>& q, const std::vector<SeedEntry>& r, std::vector<HitMap>& out,
                    size_t max_expand) {
  size_t i = 0, j = 0;
  while (i < q.size() && j < r.size()) {
    if (q[i].key < r[j].key) {
      ++i;
    } else if (q[i].key > r[j].key) {
      ++j;
    } else {
      uint64_t key = q[i].key;
      size_t qi = i, rj = j;
      while (qi < q.size() && q[qi].key == key) ++qi;
      while (rj < r.size() && r[rj].key == key) ++rj;
      if ((qi - i) * (rj - j) <= max_expand) {
        for (size_t a = i; a < qi; ++a) {
          HitMap& bucket = out[q[a].seq];
          for (size_t b = j; b < rj; ++b)
            bucket[r[b].seq].push_back(SeedHit{q[a].seq, q[a].pos, r[b].seq, r[b].pos});
        }
      }
      i = qi;
      j = rj;
    }
  }
}

std::vector<std::pair<size_t, size_t>> chunks(size_t n, size_t parts) {
  parts = std::max<size_t>(parts, 1);
  std::vector<std::pair<size_t, size_t>> out;
  if (n == 0) return out;
  parts = std::min(parts, n);
  size_t start = 0;
  for (size_t p = 0; p < parts; ++p) {
    size_t end = (p + 1 == parts) ? n : start + n / parts + (p < n % parts ? 1 : 0);
    out.emplace_back(start, end);
    start = end;
  }
  return out;
}

// --------------------------------------------------------------- ungapped.rs
Segment xdrop(const uint8_t* query, size_t qlen, const uint8_t* subject, size_t slen, size_t qa, size_t sa,
              const ScoreMatrix& m, int xd) {
  int score = 0, st = 0;
  size_t n = 1, delta = 0, len = 0;
  long q = (long)qa - 1, s = (long)sa - 1;
  while (score - st < xd && q >= 0 && s >= 0) {
    st += m.score(query[q], subject[s]);
    if (st > score) {
      score = st;
      delta = n;
    }
    --q;
    --s;
    ++n;
  }
  q = (long)qa;
  s = (long)sa;
  st = score;
  n = 1;
  while (score - st < xd && (size_t)q < qlen && (size_t)s < slen) {
    st += m.score(query[q], subject[s]);
    if (st > score) {
      score = st;
      len = n;
    }
    ++q;
    ++s;
    ++n;
  }
  return Segment{qa - delta, sa - delta, len + delta, score};
}

// ----------------------------------------------------------------- gapped.rs
size_t band_for(size_t len) {
  static const size_t THRESHOLD[7] = {50, 100, 150, 200, 250, 350, 500};
  static const size_t BAND[8] = {12, 16, 30, 30, 30, 40, 64, 64};
  size_t bucket = 0;
  for (size_t t : THRESHOLD)
    if (len >= t) ++bucket;
  return BAND[bucket];
}

void HspStats::add_match(uint8_t a, uint8_t b, const ScoreMatrix& m) {
  length += 1;
  if (a == b) identities += 1;
  else mismatches += 1;
  if (m.score(a, b) > 0) positives += 1;
}

namespace {
constexpr int32_t NEG = INT32_MIN / 4;
long clampl(long v, long lo, long hi) { return v < lo ? lo : (v > hi ? hi : v); }
}  // namespace

std::optional<Aligned> extend_span(const uint8_t* query, size_t n, const uint8_t* subject, size_t m, long d0,
                                   long d1, const ScoreMatrix& matrix, int gap_open, int gap_extend,
                                   uint64_t* cells_out) {
  if (n == 0 || m == 0) return std::nullopt;
  long lo_d = std::min(d0, d1), hi_d = std::max(d0, d1);
  d0 = lo_d;
  d1 = hi_d;
  std::vector<size_t> j0(n + 1), j1(n + 1), off(n + 2, 0);
  size_t max_w = 1;
  for (size_t i = 0; i <= n; ++i) {
    size_t lo = (size_t)clampl((long)i - d1, 0, (long)m);
    size_t hi = (size_t)clampl((long)i - d0, 0, (long)m);
    j0[i] = lo;
    j1[i] = std::max(hi, lo);
    max_w = std::max(max_w, j1[i] - j0[i] + 1);
  }
  for (size_t i = 0; i <= n; ++i) off[i + 1] = off[i] + (j1[i] - j0[i] + 1);
  std::vector<uint8_t> trace(off[n + 1], 0);
  const int open_cost = gap_open + gap_extend;
  const int ge = gap_extend;
  std::vector<int32_t> prev_h(max_w, 0), prev_e(max_w, NEG), cur_h(max_w, 0), cur_e(max_w, NEG);
  int32_t best = 0;
  size_t best_i = 0, best_j = 0;
  uint64_t cells = 0;
  for (size_t i = 1; i <= n; ++i) {
    uint8_t qi = query[i - 1];
    size_t a = j0[i], b = j1[i], pa = j0[i - 1], pb = j1[i - 1];
    int32_t f_left = NEG;
    for (size_t j = a; j <= b; ++j) {
      ++cells;
      int32_t d = NEG;
      if (j >= 1) {
        int32_t hd = (j > pa && j - 1 <= pb) ? prev_h[j - 1 - pa] : 0;
        d = hd + matrix.score(qi, subject[j - 1]);
      }
      int32_t e = NEG;
      uint8_t e_open = 0;
      if (j >= pa && j <= pb) {
        int32_t hp = prev_h[j - pa];
        if (hp > NEG / 2) {
          int32_t v = hp - open_cost;
          if (v > e) e = v;
        }
        int32_t pe = prev_e[j - pa];
        if (pe > NEG / 2) {
          int32_t v = pe - ge;
          if (v > e) {
            e = v;
            e_open = 1;
          }
        }
      }
      int32_t f = NEG;
      uint8_t f_open = 0;
      if (j > a) {
        int32_t hl = cur_h[j - 1 - a];
        if (hl > NEG / 2) {
          int32_t v = hl - open_cost;
          if (v > f) f = v;
        }
        if (f_left > NEG / 2) {
          int32_t v = f_left - ge;
          if (v > f) {
            f = v;
            f_open = 1;
          }
        }
      }
      int32_t hv = 0;
      uint8_t choice = 0;
      if (d > hv) { hv = d; choice = 1; }
      if (e > hv) { hv = e; choice = 2; }
      if (f > hv) { hv = f; choice = 3; }
      cur_h[j - a] = hv;
      cur_e[j - a] = e;
      trace[off[i] + j - a] = (uint8_t)(choice | (e_open << 2) | (f_open << 3));
      f_left = f;
      if (hv > best) {
        best = hv;
        best_i = i;
        best_j = j;
      }
    }
    std::swap(prev_h, cur_h);
    std::swap(prev_e, cur_e);
  }
  if (cells_out) *cells_out = cells;
  if (best <= 0) return std::nullopt;

  std::vector<Op> rev;
  HspStats stats;
  int state = 0;
  size_t i = best_i, j = best_j;
  bool in_gap = false;
  while (i > 0 && j > 0) {
    if (j < j0[i] || j > j1[i]) break;
    uint8_t t = trace[off[i] + j - j0[i]];
    if (state == 0) {
      int c = t & 3;
      if (c == 0) break;
      if (c == 1) {
        stats.add_match(query[i - 1], subject[j - 1], matrix);
        rev.push_back(Op::Match);
        in_gap = false;
        --i;
        --j;
      } else if (c == 2) {
        state = 1;
      } else {
        state = 2;
      }
    } else if (state == 1) {
      stats.length += 1;
      stats.gaps += 1;
      if (!in_gap) {
        stats.gap_openings += 1;
        in_gap = true;
      }
      rev.push_back(Op::Ins);
      if (((t >> 2) & 1) == 0) state = 0;
      --i;
    } else {
      stats.length += 1;
      stats.gaps += 1;
      if (!in_gap) {
        stats.gap_openings += 1;
        in_gap = true;
      }
      rev.push_back(Op::Del);
      if (((t >> 3) & 1) == 0) state = 0;
      --j;
    }
  }
  std::reverse(rev.begin(), rev.end());
  Aligned out;
  for (Op op : rev) {
    if (!out.ops.empty() && out.ops.back().first == op) out.ops.back().second += 1;
    else out.ops.emplace_back(op, 1u);
  }
  if (out.ops.empty()) return std::nullopt;
  out.score = best;
  out.q_begin = i;
  out.q_end = best_i;
  out.s_begin = j;
  out.s_end = best_j;
  out.stats = stats;
  out.cells = cells;
  return out;
}

// -------------------------------------------------------------------- hsp.rs
std::pair<size_t, size_t> Hsp::nt_range(size_t dna_len) const {  // hsp.rs:99-110
  size_t f = frame;
  if (f < 3) return {f + 3 * q_begin, f + 3 * q_end};
  size_t o = f - 3;
  return {dna_len - (o + 3 * q_end), dna_len - (o + 3 * q_begin)};
}
double Hsp::pident() const {  // hsp.rs:113-119
  return stats.length == 0 ? 0.0 : (double)stats.identities * 100.0 / (double)stats.length;
}
double Hsp::ppos() const {  // hsp.rs:122-128
  return stats.length == 0 ? 0.0 : (double)stats.positives * 100.0 / (double)stats.length;
}
static char op_code(Op o) { return o == Op::Match ? 'M' : (o == Op::Ins ? 'I' : 'D'); }
std::string Hsp::cigar() const {  // hsp.rs:152-159
  std::string out;
  for (auto& p : ops) {
    out += std::to_string(p.second);
    out += op_code(p.first);
  }
  return out;
}
std::pair<std::string, std::string> Hsp::aligned_strings(const uint8_t* q, const uint8_t* s) const {  // hsp.rs:164-192
  std::string a, b;
  size_t qi = q_begin, si = s_begin;
  for (auto& p : ops) {
    for (uint32_t k = 0; k < p.second; ++k) {
      if (p.first == Op::Match) {
        a += decode_byte(q[qi++]);
        b += decode_byte(s[si++]);
      } else if (p.first == Op::Ins) {
        a += decode_byte(q[qi++]);
        b += '-';
      } else {
        a += '-';
        b += decode_byte(s[si++]);
      }
    }
  }
  return {a, b};
}
std::string Hsp::btop(const uint8_t* q, const uint8_t* s) const {  // hsp.rs:195-241
  std::string out;
  uint32_t matches = 0;
  size_t qi = q_begin, si = s_begin;
  auto flush = [&]() {
    if (matches > 0) {
      out += std::to_string(matches);
      matches = 0;
    }
  };
  for (auto& p : ops) {
    for (uint32_t k = 0; k < p.second; ++k) {
      if (p.first == Op::Match) {
        char a = decode_byte(q[qi]), b = decode_byte(s[si]);
        if (a == b) {
          ++matches;
        } else {
          flush();
          out += a;
          out += b;
        }
        ++qi;
        ++si;
      } else if (p.first == Op::Ins) {
        flush();
        out += decode_byte(q[qi]);
        out += '-';
        ++qi;
      } else {
        flush();
        out += '-';
        out += decode_byte(s[si]);
        ++si;
      }
    }
  }
  flush();
  return out;
}

// ----------------------------------------------------------------- alp.rs
namespace {
constexpr double LN_2 = 0.693147180559945309417232121458176568;
constexpr double NAT_CUT_OFF_IN_MAX = 2.0;
constexpr double ROOT6_EPS = 2.4607833005759251e-3;
constexpr double SQRT_PI = 1.772453850905516;
constexpr double INV_SQRT_2PI = 0.3989422804014327;
constexpr double PI = 3.14159265358979323846264338327950288;
const double NEG_INF = -INFINITY;

double ln_or_neg_inf(double x) { return x > 0.0 ? std::log(x) : NEG_INF; }
double log_sum(double a, double b) {
  double hi = a >= b ? a : b, lo = a >= b ? b : a;
  if (!std::isfinite(hi)) return hi;
  if (lo == NEG_INF) return hi;
  return hi + std::log(1.0 + std::exp(lo - hi));
}
double log_diff(double a, double b) {
  if (a < b) return NEG_INF;
  if (!std::isfinite(a)) return a;
  if (b == NEG_INF) return a;
  double t = 1.0 - std::exp(b - a);
  return t <= 0.0 ? NEG_INF : a + std::log(t);
}
double cheb_eval(const double* c, int len, double x) {
  int n = len - 1;
  double y2 = 2.0 * x, d = 0.0, dd = 0.0;
  for (int j = n; j >= 1; --j) {
    double temp = d;
    d = y2 * d - dd + c[j];
    dd = temp;
  }
  return x * d - dd + 0.5 * c[0];
}
double erfc8_sum(double x) {
  double num = kErfc8P[5];
  for (int i = 4; i >= 0; --i) num = x * num + kErfc8P[i];
  double den = kErfc8Q[6];
  for (int i = 5; i >= 0; --i) den = x * den + kErfc8Q[i];
  return num / den;
}
double erfc_gsl(double x) {
  double ax = std::fabs(x), v;
  if (ax <= 1.0) v = cheb_eval(kErfcXlt1, 20, 2.0 * ax - 1.0);
  else if (ax <= 5.0) v = std::exp(-x * x) * cheb_eval(kErfcX15, 25, 0.5 * (ax - 3.0));
  else if (ax < 10.0) v = std::exp(-x * x) / ax * cheb_eval(kErfcX510, 20, (2.0 * ax - 15.0) / 5.0);
  else v = erfc8_sum(ax) * std::exp(-x * x);
  return x < 0.0 ? 2.0 - v : v;
}
}  // namespace

double log_erfc(double x) {
  if (x < -8.0) return LN_2;
  if (x * x < 10.0 * ROOT6_EPS) {
    double y = x / SQRT_PI;
    const double C3 = (4.0 - PI) / 3.0;
    const double C4 = 2.0 * (1.0 - PI / 3.0);
    const double* c = kLogErfcSeries;  // C5..C14
    double series = c[3] + y * (c[4] + y * (c[5] + y * (c[6] + y * (c[7] + y * (c[8] + c[9] * y)))));
    series = y * (1.0 + y * (1.0 + y * (C3 + y * (C4 + y * (c[0] + y * (c[1] + y * (c[2] + y * series)))))));
    return -2.0 * series;
  }
  if (x > 8.0) return std::log(erfc8_sum(x)) - x * x;
  return std::log(erfc_gsl(x));
}

AlpParams AlpParams::make(double lambda, double k, double alpha, double alpha_v, double sigma, int go, int ge,
                          double u_alpha, double u_alpha_v) {
  double g = (double)(go + ge);
  AlpParams p;
  p.lambda = lambda;
  p.k = k;
  p.a = alpha;
  p.b = 2.0 * g * (u_alpha - alpha);
  p.alpha = alpha_v;
  p.beta = 2.0 * g * (u_alpha_v - alpha_v);
  p.a_j = alpha;
  p.b_j = p.b;
  p.alpha_j = alpha_v;
  p.beta_j = p.beta;
  p.sigma = sigma;
  p.tau = 2.0 * g * (u_alpha_v - sigma);
  p.vi_thr = std::fmax(NAT_CUT_OFF_IN_MAX * alpha_v / lambda, 0.0);
  p.vj_thr = std::fmax(NAT_CUT_OFF_IN_MAX * alpha_v / lambda, 0.0);
  p.c_thr = std::fmax(NAT_CUT_OFF_IN_MAX * sigma / lambda, 0.0);
  return p;
}

double AlpParams::blast_evalue(int raw, size_t qlen, uint64_t db) const {
  double exponent = -lambda * (double)raw + std::log(k);
  if (exponent > 700.0) return INFINITY;
  return (double)qlen * (double)db * std::exp(exponent);
}

double AlpParams::evalue(int raw, size_t qlen, size_t slen, uint64_t db) const {
  double y = (double)raw;
  double m = (double)std::max<size_t>(slen, 1);
  double n = (double)std::max<size_t>(qlen, 1);
  double la = log_area(y, m, n);
  if (!std::isfinite(la)) return blast_evalue(raw, qlen, db);
  double log_e = la + std::log(k) - lambda * y;
  if (log_e > 700.0) return INFINITY;
  return std::exp(log_e) * (double)db / m;
}

double AlpParams::log_area(double y, double m, double n) const {
  double m_li_y = m - (a * y + b);
  double vi_y = std::fmax(vi_thr, alpha * y + beta);
  double sqrt_vi = std::sqrt(vi_y);
  double m_f = sqrt_vi == 0.0 ? 1e100 : m_li_y / sqrt_vi;
  double log_p_m = std::log(0.5) + log_erfc(-std::sqrt(0.5) * m_f);
  double log_e_m = std::log(INV_SQRT_2PI) - 0.5 * m_f * m_f;
  double log_sqrt_e_m = ln_or_neg_inf(sqrt_vi) + log_e_m;
  double log_p1 = m_li_y < 0.0 ? log_diff(log_sqrt_e_m, ln_or_neg_inf(-m_li_y) + log_p_m)
                               : log_sum(log_sqrt_e_m, ln_or_neg_inf(m_li_y) + log_p_m);
  double n_lj_y = n - (a_j * y + b_j);
  double vj_y = std::fmax(vj_thr, alpha_j * y + beta_j);
  double sqrt_vj = std::sqrt(vj_y);
  double n_f = sqrt_vj == 0.0 ? 1e100 : n_lj_y / sqrt_vj;
  double log_p_n = std::log(0.5) + log_erfc(-std::sqrt(0.5) * n_f);
  double log_e_n = std::log(INV_SQRT_2PI) - 0.5 * n_f * n_f;
  double log_sqrt_e_n = ln_or_neg_inf(sqrt_vj) + log_e_n;
  double log_p2 = n_lj_y < 0.0 ? log_diff(log_sqrt_e_n, ln_or_neg_inf(-n_lj_y) + log_p_n)
                               : log_sum(log_sqrt_e_n, ln_or_neg_inf(n_lj_y) + log_p_n);
  double c_y = std::fmax(c_thr, sigma * y + tau);
  double log_c_y = ln_or_neg_inf(c_y);
  return log_sum(log_p1 + log_p2, log_c_y + log_p_m + log_p_n);
}

// --------------------------------------------------------------- matrix.rs
bool score_matrix_standard(const std::string& name, int go, int ge, ScoreMatrix* out, std::string* err) {
  std::string upper = name;
  for (auto& c : upper) c = (char)toupper((unsigned char)c);
  const StdMatrixDef* def = nullptr;
  for (int i = 0; i < kNumStdMatrices; ++i)
    if (upper == kStdMatrices[i].name) def = &kStdMatrices[i];
  if (!def) {
    *err = "Unknown scoring matrix: " + name;
    return false;
  }
  if (go == -1) go = def->default_go;
  if (ge == -1) ge = def->default_ge;
  if (go <= 0 || ge <= 0) {
    *err = "gap penalties must be positive (got " + std::to_string(go) + "/" + std::to_string(ge) + ")";
    return false;
  }
  const StdParamRow* row = nullptr;
  for (int i = 0; i < def->n_params; ++i)
    if (def->params[i].go == go && def->params[i].ge == ge) row = &def->params[i];
  if (!row) {
    *err = std::string("Gap penalty settings are outside the supported range for ") + def->name + " (--gapopen " +
           std::to_string(go) + " --gapextend " + std::to_string(ge) + ").";
    return false;
  }
  ScoreMatrix m;
  m.name = def->name;
  for (int i = 0; i < 625; ++i) m.scores[i] = def->scores[i];
  m.gap_open = go;
  m.gap_extend = ge;
  m.lambda = row->lambda;
  m.k = row->k;
  m.ln_k = std::log(row->k);
  m.has_alp = true;
  m.alp = AlpParams::make(row->lambda, row->k, row->alpha, row->alpha_v, row->sigma, go, ge, def->u_alpha,
                          def->u_alpha_v);
  *out = m;
  return true;
}

int ScoreMatrix::raw_score(double bits) const { return (int)std::ceil((bits * LN_2 + ln_k) / lambda); }
double ScoreMatrix::bit_score(int raw) const { return (lambda * (double)raw - ln_k) / LN_2; }
double ScoreMatrix::evalue(int raw, size_t qlen, size_t slen, uint64_t db) const {
  return has_alp ? alp.evalue(raw, qlen, slen, db) : evalue_blast(raw, qlen, db);
}
double ScoreMatrix::evalue_blast(int raw, size_t qlen, uint64_t db) const {
  double exponent = -lambda * (double)raw + ln_k;
  if (exponent > 700.0) return INFINITY;
  return (double)qlen * (double)db * std::exp(exponent);
}

}  // namespace oracle
