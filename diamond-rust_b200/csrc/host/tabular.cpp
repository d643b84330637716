#include "tabular.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>

namespace drg {
namespace host {

// ---- output.rs ----------------------------------------------------------------------
namespace {
const char* kFieldNames[] = {"qseqid", "qlen", "sseqid", "slen", "qstart", "qend", "sstart", "send", "qseq",
                             "sseq", "evalue", "bitscore", "score", "length", "pident", "nident", "mismatch",
                             "positive", "gapopen", "gaps", "ppos", "qframe", "qcovhsp", "scovhsp", "cigar",
                             "btop", "qtitle", "stitle", "full_sseq", "qseq_translated", "qstrand"};
const std::vector<Field> kDefaultFields = {kQSeqId, kSSeqId, kPIdent, kLength,
                                           kMismatch, kGapOpen, kQStart, kQEnd, kSStart, kSEnd, kEValue,
                                           kBitScore};

// Rust's Debug rendering of a string argument ("{other:?}") for plain ASCII.
std::string debug_quote(const std::string& s) {
  std::string o = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') o.push_back('\\');
    o.push_back(c);
  }
  return o + "\"";
}
}  // namespace

std::vector<Field> parse_outfmt_tokens(const std::vector<std::string>& tokens) {
  if (tokens.empty()) return kDefaultFields;
  const std::string& first = tokens[0];
  if (first == "0" || first == "5" || first == "102")
    throw std::runtime_error("--outfmt " + first + " is not supported, use 6 (tabular)");
  if (first != "6") throw std::runtime_error("invalid --outfmt value " + debug_quote(first));
  if (tokens.size() <= 1) return kDefaultFields;
  std::vector<Field> f;
  for (size_t i = 1; i < tokens.size(); ++i) {
    int k = -1;
    for (int j = 0; j < (int)(sizeof kFieldNames / sizeof kFieldNames[0]); ++j)
      if (tokens[i] == kFieldNames[j]) k = j;
    if (k < 0) throw std::runtime_error("Invalid output field: " + tokens[i]);
    f.push_back((Field)k);
  }
  return f;
}

std::string format_double(double x) {
  char b[64];
  if (x >= 100.0) return std::to_string((long long)std::floor(x));
  std::snprintf(b, sizeof b, "%.1f", x);
  return b;
}

std::string format_evalue(double e) {
  if (!std::isfinite(e) || e <= 0.0) return "0.0";
  char b[64];
  std::snprintf(b, sizeof b, "%.2e", e);  // d.dde[+-]XX
  std::string s(b);
  const size_t p = s.find('e');
  const int ex = std::atoi(s.c_str() + p + 1);
  return s.substr(0, p + 1) + std::to_string(ex);  // Rust prints the bare exponent
}

std::string tabular_row(const drg_hsp& h, const uint32_t* ops, const QueryView& q, const DbFile& db,
                        const std::vector<Field>& fields) {
  const uint8_t* subject = db.seq(h.subject);
  const uint64_t slen = db.seq_len(h.subject);
  const uint64_t f = h.frame;
  uint64_t qb = h.q_begin, qe = h.q_end;
  if (q.translated) {  // hsp.rs:97-109 nt_range
    if (f < 3) {
      qb = f + 3ull * h.q_begin;
      qe = f + 3ull * h.q_end;
    } else {
      const uint64_t o = f - 3;
      qb = q.dna_len - (o + 3ull * h.q_end);
      qe = q.dna_len - (o + 3ull * h.q_begin);
    }
  }
  const uint64_t qlen = q.translated ? q.dna_len : q.frame_len;
  auto pct = [](uint32_t a, uint32_t len) { return len == 0 ? 0.0 : (double)a * 100.0 / (double)len; };
  auto aligned = [&](bool want_q) {
    std::string s;
    uint64_t qi = h.q_begin, si = h.s_begin;
    for (uint32_t k = 0; k < h.n_ops; ++k) {
      const uint32_t op = ops[k] & 3u, n = ops[k] >> 2;
      for (uint32_t r = 0; r < n; ++r) {
        if (op == 0) {
          s.push_back(want_q ? decode_letter(q.letters[qi]) : decode_letter(subject[si]));
          ++qi;
          ++si;
        } else if (op == 1) {
          s.push_back(want_q ? decode_letter(q.letters[qi]) : '-');
          ++qi;
        } else {
          s.push_back(want_q ? '-' : decode_letter(subject[si]));
          ++si;
        }
      }
    }
    return s;
  };
  std::string row;
  for (size_t fi = 0; fi < fields.size(); ++fi) {
    if (fi) row.push_back('\t');
    switch (fields[fi]) {
      case kQSeqId: row += *q.id; break;
      case kQLen: row += std::to_string(qlen); break;
      case kSSeqId: row += db.id(h.subject); break;
      case kSLen: row += std::to_string(slen); break;
      case kQStart: row += std::to_string(qb + 1); break;
      case kQEnd: row += std::to_string(qe); break;
      case kSStart: row += std::to_string((uint64_t)h.s_begin + 1); break;
      case kSEnd: row += std::to_string(h.s_end); break;
      case kQSeq: row += aligned(true); break;
      case kSSeq: row += aligned(false); break;
      case kEValue: row += format_evalue(h.evalue); break;
      case kBitScore: row += format_double(h.bits); break;
      case kScore: row += std::to_string(h.score); break;
      case kLength: row += std::to_string(h.length); break;
      case kPIdent: row += format_double(pct(h.identities, h.length)); break;
      case kNIdent: row += std::to_string(h.identities); break;
      case kMismatch: row += std::to_string(h.mismatches); break;
      case kPositive: row += std::to_string(h.positives); break;
      case kGapOpen: row += std::to_string(h.gap_openings); break;
      case kGaps: row += std::to_string(h.gaps); break;
      case kPPos: row += format_double(pct(h.positives, h.length)); break;
      case kQFrame: row += std::to_string(f < 3 ? (long long)f + 1 : 2 - (long long)f); break;
      case kQCovHsp:
        row += qlen == 0 ? "0.0" : format_double((double)(qe - qb) * 100.0 / (double)qlen);
        break;
      case kSCovHsp:
        row += slen == 0 ? "0.0" : format_double((double)(h.s_end - h.s_begin) * 100.0 / (double)slen);
        break;
      case kCigar:
        for (uint32_t k = 0; k < h.n_ops; ++k) {
          row += std::to_string(ops[k] >> 2);
          row.push_back("MID"[ops[k] & 3u]);
        }
        break;
      case kBTop: {  // hsp.rs:181-239
        uint32_t run = 0;
        uint64_t qi = h.q_begin, si = h.s_begin;
        auto flush = [&]() {
          if (run) row += std::to_string(run);
          run = 0;
        };
        for (uint32_t k = 0; k < h.n_ops; ++k) {
          const uint32_t op = ops[k] & 3u, n = ops[k] >> 2;
          for (uint32_t r = 0; r < n; ++r) {
            if (op == 0) {
              const char a = decode_letter(q.letters[qi++]), b = decode_letter(subject[si++]);
              if (a == b) {
                ++run;
              } else {
                flush();
                row.push_back(a);
                row.push_back(b);
              }
            } else if (op == 1) {
              flush();
              row.push_back(decode_letter(q.letters[qi++]));
              row.push_back('-');
            } else {
              flush();
              row.push_back('-');
              row.push_back(decode_letter(subject[si++]));
            }
          }
        }
        flush();
        break;
      }
      case kQTitle: row += *q.header; break;
      case kSTitle: row += db.header(h.subject); break;
      case kFullSSeq: row += decode_residues(subject, slen); break;
      case kQSeqTranslated: {
        const uint64_t end = std::min<uint64_t>(h.q_end, q.frame_len);
        const uint64_t begin = std::min<uint64_t>(h.q_begin, end);
        row += decode_residues(q.letters + begin, end - begin);
        break;
      }
      case kQStrand: row += f >= 3 ? "-" : "+"; break;
    }
  }
  return row;
}

}  // namespace host
}  // namespace drg
