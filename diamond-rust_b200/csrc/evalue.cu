// E-value gate and per-pair band walk (search.rs:232-255) on the device.
//
// The reference keeps a band's HSP when its ALP E-value (alp.rs:108-163) is
// <= --evalue, walking a pair's bands in order until --max-hsps are kept.
// The device evaluates the same formula in double precision with CUDA's
// libm; its last bits can differ from the host's glibc, so a band is decided
// here only when the device value is clear of the threshold by a relative
// margin of 1e-9 (orders of magnitude above the error of either libm).  A
// pair that meets an undecided band is handed back to the host, which redoes
// its walk with the exact host statistics.
#include <mutex>

#include "kernels.h"

namespace drg {

namespace {
#include "host/score_tables.inc"
}  // namespace

__constant__ double c_xlt1[20], c_x15[25], c_x510[20], c_p8[6], c_q8[7], c_ser[10];
// The tables are the same for every search: copied once per device, with a
// blocking copy under a lock, before any context's first E-value launch.
static std::mutex g_alp_mutex;
static bool g_alp_ready[64] = {};

void upload_alp_tables(cudaStream_t) {
  int dev = 0;
  DRG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_alp_mutex);
  if (dev < 0 || dev >= 64 || g_alp_ready[dev]) return;
  DRG_CUDA(cudaMemcpyToSymbol(c_xlt1, kErfcXlt1, sizeof(kErfcXlt1)));
  DRG_CUDA(cudaMemcpyToSymbol(c_x15, kErfcX15, sizeof(kErfcX15)));
  DRG_CUDA(cudaMemcpyToSymbol(c_x510, kErfcX510, sizeof(kErfcX510)));
  DRG_CUDA(cudaMemcpyToSymbol(c_p8, kErfc8P, sizeof(kErfc8P)));
  DRG_CUDA(cudaMemcpyToSymbol(c_q8, kErfc8Q, sizeof(kErfc8Q)));
  DRG_CUDA(cudaMemcpyToSymbol(c_ser, kLogErfcSeries, sizeof(kLogErfcSeries)));
  g_alp_ready[dev] = true;
}

namespace {
__device__ double d_clenshaw(const double* c, int len, double x) {
  double two_x = 2.0 * x, b1 = 0.0, b2 = 0.0;
  for (int k = len - 1; k >= 1; --k) {
    double t = b1;
    b1 = two_x * b1 - b2 + c[k];
    b2 = t;
  }
  return x * b1 - b2 + 0.5 * c[0];
}
__device__ double d_tail(double x) {
  double p = c_p8[5];
  for (int i = 4; i >= 0; --i) p = x * p + c_p8[i];
  double q = c_q8[6];
  for (int i = 5; i >= 0; --i) q = x * q + c_q8[i];
  return p / q;
}
__device__ double d_log_erfc(double x) {
  if (x < -8.0) return 0.693147180559945309417232121458176568;
  if (x * x < 10.0 * 2.4607833005759251e-3) {
    const double pi = 3.14159265358979323846264338327950288;
    double y = x / 1.772453850905516;
    double c3 = (4.0 - pi) / 3.0, c4 = 2.0 * (1.0 - pi / 3.0);
    const double* c = c_ser;
    double s = c[3] + y * (c[4] + y * (c[5] + y * (c[6] + y * (c[7] + y * (c[8] + c[9] * y)))));
    s = y * (1.0 + y * (1.0 + y * (c3 + y * (c4 + y * (c[0] + y * (c[1] + y * (c[2] + y * s)))))));
    return -2.0 * s;
  }
  if (x > 8.0) return log(d_tail(x)) - x * x;
  double ax = fabs(x), r;
  if (ax <= 1.0) r = d_clenshaw(c_xlt1, 20, 2.0 * ax - 1.0);
  else if (ax <= 5.0) r = exp(-x * x) * d_clenshaw(c_x15, 25, 0.5 * (ax - 3.0));
  else if (ax < 10.0) r = exp(-x * x) / ax * d_clenshaw(c_x510, 20, (2.0 * ax - 15.0) / 5.0);
  else r = d_tail(ax) * exp(-x * x);
  return log(x < 0.0 ? 2.0 - r : r);
}
__device__ double d_log_pos(double x) { return x > 0.0 ? log(x) : -INFINITY; }
__device__ double d_log_add(double a, double b) {
  double hi = a >= b ? a : b, lo = a >= b ? b : a;
  if (!isfinite(hi) || lo == -INFINITY) return hi;
  return hi + log(1.0 + exp(lo - hi));
}
__device__ double d_log_sub(double a, double b) {
  if (a < b) return -INFINITY;
  if (!isfinite(a) || b == -INFINITY) return a;
  double t = 1.0 - exp(b - a);
  return t <= 0.0 ? -INFINITY : a + log(t);
}
__device__ double d_log_axis(double len, double y, const AlpDev& A, double* log_p) {
  double l = len - (A.a * y + A.b);
  double v = fmax(A.v_thr, A.alpha * y + A.beta);
  double sv = sqrt(v);
  double z = sv == 0.0 ? 1e100 : l / sv;
  *log_p = log(0.5) + d_log_erfc(-sqrt(0.5) * z);
  double lsp = d_log_pos(sv) + (log(0.3989422804014327) - 0.5 * z * z);
  return l < 0.0 ? d_log_sub(lsp, d_log_pos(-l) + *log_p) : d_log_add(lsp, d_log_pos(l) + *log_p);
}
}  // namespace

__device__ double alp_evalue_dev(const AlpDev& A, int raw, uint64_t qlen, uint64_t slen, uint64_t db) {
  double y = (double)raw;
  double m = (double)(slen > 0 ? slen : 1), n = (double)(qlen > 0 ? qlen : 1);
  double lpm, lpn;
  double l1 = d_log_axis(m, y, A, &lpm);
  double l2 = d_log_axis(n, y, A, &lpn);
  double c = fmax(A.c_thr, A.sigma * y + A.tau);
  double la = d_log_add(l1 + l2, d_log_pos(c) + lpm + lpn);
  if (!isfinite(la)) {
    double e = -A.lambda * y + A.ln_k;
    return e > 700.0 ? INFINITY : (double)qlen * (double)db * exp(e);
  }
  double le = la + A.ln_k - A.lambda * y;
  return le > 700.0 ? INFINITY : exp(le) * (double)db / m;
}

// sum over rows i = 1..n of clamp(i - d0, 0, m) - clamp(i - d1, 0, m) + 1, the
// reference's row ranges (gapped.rs:82-93), in closed form: with
// G(t) = sum_{x=0..t} clamp(x, 0, m), sum_{i=1..n} clamp(i - d, 0, m) is
// G(n - d) - G(-d).
__host__ __device__ __forceinline__ int64_t clamp_prefix(int64_t t, int64_t m) {
  if (t < 0) return 0;
  if (t <= m) return t * (t + 1) / 2;
  return m * (m + 1) / 2 + (t - m) * m;
}
__host__ __device__ uint64_t band_cells(uint32_t n, uint32_t m, int32_t d0, int32_t d1) {
  const int64_t N = n, M = m;
  const int64_t s0 = clamp_prefix(N - d0, M) - clamp_prefix(-(int64_t)d0, M);
  const int64_t s1 = clamp_prefix(N - d1, M) - clamp_prefix(-(int64_t)d1, M);
  return (uint64_t)(s0 - s1 + N);
}
uint64_t band_cells_host(uint32_t n, uint32_t m, int32_t d0, int32_t d1) { return band_cells(n, m, d0, d1); }

namespace {
// E-value verdict of every band: 1 fails, 2 passes, 3 too close to the
// threshold to decide on the device (the host ALP settles it).  Independent per
// band (it depends on score, qlen, slen only), so one thread per band.
__global__ void k_band_verdict(SelectArgs a) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= a.n_bands) return;
  const int sc = a.score[i];
  if (sc <= 0) {
    a.verdict[i] = 1;
    return;
  }
  const Band bd = a.bands[i];
  const uint32_t slen = (uint32_t)(a.s_offsets[bd.subject + 1] - a.s_offsets[bd.subject]);
  const uint64_t qlen = a.q_offsets[bd.target + 1] - a.q_offsets[bd.target];
  const double lo_thr = a.evalue * (1.0 - 1e-9), hi_thr = a.evalue * (1.0 + 1e-9);
  const double ev = alp_evalue_dev(a.alp, sc, qlen, slen, a.db_letters);
  a.verdict[i] = ev <= lo_thr ? 2 : ((ev > hi_thr || isnan(ev)) ? 1 : 3);
}

// The reference's walk over a pair's bands in rank order (search.rs:233-255):
// bands are computed until max_hsps pass; an undecided verdict stops the
// device walk and leaves the rest of the pair to the host.
__global__ void k_select(SelectArgs a) {
  const uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  // threads past the last pair walk an empty range and join the reduction
  const uint64_t b = p < a.n_pairs ? a.pair_first[p] : 0, e = p < a.n_pairs ? a.pair_first[p + 1] : 0;
  uint32_t kept = 0;
  bool undecided = false;
  unsigned long long cells = 0, computed = 0;
  for (uint64_t i = b; i < e; ++i) {
    if (undecided) {
      a.state[i] = 3;
      continue;
    }
    if (kept >= a.max_hsps) {
      a.state[i] = 0;
      continue;
    }
    const Band bd = a.bands[i];
    const uint32_t slen = (uint32_t)(a.s_offsets[bd.subject + 1] - a.s_offsets[bd.subject]);
    cells += band_cells(bd.n, slen, bd.d0, bd.d1);
    ++computed;
    const uint8_t v = a.verdict[i];
    a.state[i] = v;
    if (v == 2) ++kept;
    else if (v == 3) undecided = true;
  }
  warp_sum_atomic(a.cells_ref, cells);
  warp_sum_atomic(a.n_computed, computed);
}
}  // namespace

void launch_select(const SelectArgs& a, cudaStream_t st) {
  if (a.n_pairs == 0) return;
  if (a.n_bands > 0) {
    count_launch();
    k_band_verdict<<<ceil_div(a.n_bands, 128), 128, 0, st>>>(a);
  }
  count_launch();
  k_select<<<ceil_div(a.n_pairs, 128), 128, 0, st>>>(a);
  DRG_CUDA(cudaGetLastError());
}

}  // namespace drg
