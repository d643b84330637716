// Scoring system of the search: 25x25 substitution scores, affine gap costs,
// Karlin-Altschul lambda/K and DIAMOND's ALP finite-size-corrected E-value.
// Host double-precision code; it must agree bit for bit with diamond-rust
// (matrix.rs:42-200, alp.rs:60-237), so every operation is written in the
// reference's evaluation order and the build disables FMA contraction.
#pragma once
#include <cstdint>
#include <string>

namespace drg {

struct Alp {
  double lambda, k, ln_k;
  double a, b, alpha, beta, sigma, tau, v_thr, c_thr;
  double log_area(double y, double m, double n) const;
  double evalue(int raw, uint64_t qlen, uint64_t slen, uint64_t db_letters) const;
  double blast_evalue(int raw, uint64_t qlen, uint64_t db_letters) const;
};

struct Scoring {
  std::string name;
  int8_t scores[625];  // row-major [a * 25 + b], NCBI letter order
  int gap_open = 0, gap_extend = 0;
  int max_score = 0;   // largest entry, for 16-bit overflow bounds
  Alp alp;
  int score(uint8_t a, uint8_t b) const { return scores[(a < 24 ? a : 24) * 25 + (b < 24 ? b : 24)]; }
  int raw_score(double bits) const;     // matrix.rs:182-184
  double bit_score(int raw) const;      // matrix.rs:187-189
  double evalue(int raw, uint64_t qlen, uint64_t slen, uint64_t db) const { return alp.evalue(raw, qlen, slen, db); }
};

// ScoreMatrix::standard (matrix.rs:42-98): -1 gap values select the matrix default.
bool make_scoring(const char* name, int gap_open, int gap_extend, Scoring* out, std::string* err);

// GSL's log(erfc(x)) as used by the ALP statistics (alp.rs:209-237).
double log_erfc(double x);

}  // namespace drg
