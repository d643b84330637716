// Scoring system: see scoring.h.  Built with -ffp-contract=off.
#include "scoring.h"

#include <cctype>
#include <cmath>
#include <limits>

namespace drg {

#include "score_tables.inc"

namespace {
const double kLn2 = 0.693147180559945309417232121458176568;
const double kPi = 3.14159265358979323846264338327950288;
const double kNegInf = -std::numeric_limits<double>::infinity();
const double kInf = std::numeric_limits<double>::infinity();

// Chebyshev series sum_k c_k T_k(x) with the half-weight first term (Clenshaw).
double clenshaw(const double* c, int len, double x) {
  double two_x = 2.0 * x, b1 = 0.0, b2 = 0.0;
  for (int k = len - 1; k >= 1; --k) {
    double t = b1;
    b1 = two_x * b1 - b2 + c[k];
    b2 = t;
  }
  return x * b1 - b2 + 0.5 * c[0];
}

// Rational approximation of erfc(x) * exp(x^2) for large x.
double erfc_scaled_tail(double x) {
  double p = kErfc8P[5];
  for (int i = 4; i >= 0; --i) p = x * p + kErfc8P[i];
  double q = kErfc8Q[6];
  for (int i = 5; i >= 0; --i) q = x * q + kErfc8Q[i];
  return p / q;
}

double erfc_cheb(double x) {
  double ax = std::fabs(x), r;
  if (ax <= 1.0) {
    r = clenshaw(kErfcXlt1, 20, 2.0 * ax - 1.0);
  } else if (ax <= 5.0) {
    r = std::exp(-x * x) * clenshaw(kErfcX15, 25, 0.5 * (ax - 3.0));
  } else if (ax < 10.0) {
    r = std::exp(-x * x) / ax * clenshaw(kErfcX510, 20, (2.0 * ax - 15.0) / 5.0);
  } else {
    r = erfc_scaled_tail(ax) * std::exp(-x * x);
  }
  return x < 0.0 ? 2.0 - r : r;
}

double log_pos(double x) { return x > 0.0 ? std::log(x) : kNegInf; }

double log_add(double a, double b) {  // log(e^a + e^b)
  double hi = a >= b ? a : b, lo = a >= b ? b : a;
  if (!std::isfinite(hi) || lo == kNegInf) return hi;
  return hi + std::log(1.0 + std::exp(lo - hi));
}

double log_sub(double a, double b) {  // log(e^a - e^b), -inf when not positive
  if (a < b) return kNegInf;
  if (!std::isfinite(a) || b == kNegInf) return a;
  double t = 1.0 - std::exp(b - a);
  return t <= 0.0 ? kNegInf : a + std::log(t);
}

// One length axis of the ALP area: log of the expected effective length.
double log_axis(double len, double y, double a, double b, double alpha, double beta, double v_thr,
                double* log_p_out) {
  double l = len - (a * y + b);
  double v = std::fmax(v_thr, alpha * y + beta);
  double sv = std::sqrt(v);
  double z = sv == 0.0 ? 1e100 : l / sv;
  double log_p = std::log(0.5) + log_erfc(-std::sqrt(0.5) * z);
  double log_phi = std::log(0.3989422804014327) - 0.5 * z * z;
  double log_svphi = log_pos(sv) + log_phi;
  *log_p_out = log_p;
  return l < 0.0 ? log_sub(log_svphi, log_pos(-l) + log_p) : log_add(log_svphi, log_pos(l) + log_p);
}
}  // namespace

double log_erfc(double x) {
  if (x < -8.0) return kLn2;  // erfc(x) rounds to 2
  const double root6_eps = 2.4607833005759251e-3;
  if (x * x < 10.0 * root6_eps) {  // Taylor series about 0
    double y = x / 1.772453850905516;
    const double c3 = (4.0 - kPi) / 3.0;
    const double c4 = 2.0 * (1.0 - kPi / 3.0);
    const double* c = kLogErfcSeries;  // c5 .. c14
    double s = c[3] + y * (c[4] + y * (c[5] + y * (c[6] + y * (c[7] + y * (c[8] + c[9] * y)))));
    s = y * (1.0 + y * (1.0 + y * (c3 + y * (c4 + y * (c[0] + y * (c[1] + y * (c[2] + y * s)))))));
    return -2.0 * s;
  }
  if (x > 8.0) return std::log(erfc_scaled_tail(x)) - x * x;
  return std::log(erfc_cheb(x));
}

double Alp::log_area(double y, double m, double n) const {
  double log_pm, log_pn;
  double l1 = log_axis(m, y, a, b, alpha, beta, v_thr, &log_pm);
  double l2 = log_axis(n, y, a, b, alpha, beta, v_thr, &log_pn);
  double c = std::fmax(c_thr, sigma * y + tau);
  return log_add(l1 + l2, log_pos(c) + log_pm + log_pn);
}

double Alp::blast_evalue(int raw, uint64_t qlen, uint64_t db) const {
  double e = -lambda * (double)raw + std::log(k);
  if (e > 700.0) return kInf;
  return (double)qlen * (double)db * std::exp(e);
}

double Alp::evalue(int raw, uint64_t qlen, uint64_t slen, uint64_t db) const {
  double y = (double)raw;
  double m = (double)(slen > 0 ? slen : 1);
  double n = (double)(qlen > 0 ? qlen : 1);
  double la = log_area(y, m, n);
  if (!std::isfinite(la)) return blast_evalue(raw, qlen, db);
  double le = la + std::log(k) - lambda * y;
  if (le > 700.0) return kInf;
  return std::exp(le) * (double)db / m;
}

int Scoring::raw_score(double bits) const { return (int)std::ceil((bits * kLn2 + alp.ln_k) / alp.lambda); }
double Scoring::bit_score(int raw) const { return (alp.lambda * (double)raw - alp.ln_k) / kLn2; }

bool make_scoring(const char* name, int go, int ge, Scoring* out, std::string* err) {
  std::string up = name ? name : "BLOSUM62";
  for (auto& ch : up) ch = (char)std::toupper((unsigned char)ch);
  const StdMatrixDef* def = nullptr;
  for (int i = 0; i < kNumStdMatrices; ++i)
    if (up == kStdMatrices[i].name) def = &kStdMatrices[i];
  if (!def) {
    *err = std::string("Unknown scoring matrix: ") + (name ? name : "");
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
  Scoring s;
  s.name = def->name;
  s.max_score = -128;
  for (int i = 0; i < 625; ++i) {
    s.scores[i] = def->scores[i];
    if (def->scores[i] > s.max_score) s.max_score = def->scores[i];
  }
  s.gap_open = go;
  s.gap_extend = ge;
  // ALP parameters derived from the gapped row and the ungapped (alpha, alpha_v)
  // exactly as alp_params() does (alp.rs:60-92): both length axes share them.
  double g = (double)(go + ge);
  Alp& a = s.alp;
  a.lambda = row->lambda;
  a.k = row->k;
  a.ln_k = std::log(row->k);
  a.a = row->alpha;
  a.b = 2.0 * g * (def->u_alpha - row->alpha);
  a.alpha = row->alpha_v;
  a.beta = 2.0 * g * (def->u_alpha_v - row->alpha_v);
  a.sigma = row->sigma;
  a.tau = 2.0 * g * (def->u_alpha_v - row->sigma);
  a.v_thr = std::fmax(2.0 * row->alpha_v / row->lambda, 0.0);
  a.c_thr = std::fmax(2.0 * row->sigma / row->lambda, 0.0);
  *out = s;
  return true;
}

}  // namespace drg
