// The C ABI (include/drgpu.h): argument checks, error mapping, and the stage
// entry points (seed::build, seed::join_into, ungapped::xdrop,
// gapped::extend_span) built from the same kernels as the search.
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <unordered_map>

#include "context.h"
#include "kernels.h"

using namespace drg;

namespace {
std::atomic<uint64_t> g_launches{0};
}  // namespace

namespace drg {
// The message drg_last_error returns, from host code that sees the context
// only through the C ABI (the per-stage search).
void set_context_error(drg_ctx* ctx, const std::string& msg) {
  if (ctx) ctx->err = msg;
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t kernel_launch_count() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace drg

namespace {

#define API_BEGIN(ctx) \
  try {                \
    if (ctx) DRG_CUDA(cudaSetDevice((ctx)->device));
#define API_END(ctx)                                   \
  }                                                    \
  catch (const drg::Error& e) {                        \
    if (ctx) (ctx)->err = e.what();                    \
    return e.code;                                     \
  }                                                    \
  catch (const std::bad_alloc&) {                      \
    if (ctx) (ctx)->err = "host allocation failed";    \
    return DRG_ERR_OOM;                                \
  }                                                    \
  catch (const std::exception& e) {                    \
    if (ctx) (ctx)->err = e.what();                    \
    return DRG_ERR_INVALID;                            \
  }                                                    \
  return DRG_OK;

// Device copy of a sequence set with its letter -> sequence map.
struct Seqs {
  uint8_t* letters = nullptr;
  uint8_t* score_letters = nullptr;  // clamped to 24 for the DP kernels, when some code is above 24
  uint64_t* offsets = nullptr;
  uint32_t* owner = nullptr;
  std::vector<uint64_t> h_offsets;
  uint64_t n = 0, total = 0;
  Seqs() = default;
  Seqs(const Seqs&) = delete;
  ~Seqs() {
    cudaFree(letters);
    cudaFree(score_letters);
    cudaFree(offsets);
    cudaFree(owner);
  }
  void upload(drg_ctx* c, const uint8_t* l, const uint64_t* off, uint64_t count) {
    n = count;
    h_offsets.assign(off, off + n + 1);
    total = off[n];
    for (uint64_t i = 0; i < n; ++i)
      if (off[i + 1] < off[i]) throw Error(DRG_ERR_INVALID, "offsets must be non-decreasing");
    DRG_CUDA(cudaMalloc(&letters, total + 64));
    DRG_CUDA(cudaMalloc(&offsets, (n + 1) * sizeof(uint64_t)));
    DRG_CUDA(cudaMalloc(&owner, (total + 1) * sizeof(uint32_t)));
    DRG_CUDA(cudaMemsetAsync(letters + total, 25, 64, c->stream));
    if (total) DRG_CUDA(cudaMemcpyAsync(letters, l, total, cudaMemcpyHostToDevice, c->stream));
    DRG_CUDA(cudaMemcpyAsync(offsets, off, (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    launch_letter_owner(offsets, n, 0, total, owner, c->stream);
    if (letters_above_24(c, letters, total)) {
      DRG_CUDA(cudaMalloc(&score_letters, total + 64));
      DRG_CUDA(cudaMemsetAsync(score_letters + total, 25, 64, c->stream));
      launch_clamp_letters(letters, total, score_letters, c->stream);
    }
  }
  DevSeqs view() const { return DevSeqs{letters, offsets, &h_offsets, score_letters}; }
};

template <typename T>
struct DevArr {
  T* p = nullptr;
  DevArr() = default;
  explicit DevArr(size_t n) { DRG_CUDA(cudaMalloc(&p, (n ? n : 1) * sizeof(T))); }
  DevArr(const DevArr&) = delete;
  ~DevArr() { cudaFree(p); }
};

template <typename F>
void cub_run(drg_ctx* c, F f) {
  size_t bytes = 0;
  DRG_CUDA(f(nullptr, bytes));
  void* t = c->cub_tmp.ensure(bytes);
  DRG_CUDA(f(t, bytes));
}

// Waits for the context's stream; a radix sort whose bounded wait gave up
// since the last check makes the call fail.
void sync(drg_ctx* c) {
  uint32_t* d_err = c->sort_err.as<uint32_t>(1);
  uint32_t* h = c->h_stage.as<uint32_t>(1);
  DRG_CUDA(cudaMemcpyAsync(h, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  DRG_CUDA(cudaStreamSynchronize(c->stream));
  if (*h) {
    DRG_CUDA(cudaMemsetAsync(d_err, 0, sizeof(uint32_t), c->stream));
    throw Error(DRG_ERR_TIMEOUT, "radix sort: a tile's bounded wait for an earlier tile gave up");
  }
}

int cmp_hsp(const drg_hsp& a, const drg_hsp& b) {  // search.rs:273-282
  if (a.score != b.score) return b.score < a.score ? -1 : 1;
  if (a.evalue < b.evalue) return -1;
  if (a.evalue > b.evalue) return 1;
  if (a.subject != b.subject) return a.subject < b.subject ? -1 : 1;
  return 0;
}

}  // namespace

extern "C" {

const char* drg_version(void) { return "drgpu 0.1 (sm_100a)"; }

void drg_free(void* p) { std::free(p); }

// Constant-memory banks in use, one per live context.
static std::mutex g_slot_mutex;
static bool g_slot_used[kConstSlots] = {};
static int acquire_slot() {
  std::lock_guard<std::mutex> lock(g_slot_mutex);
  for (int i = 0; i < kConstSlots; ++i)
    if (!g_slot_used[i]) {
      g_slot_used[i] = true;
      return i;
    }
  return -1;
}
static void release_slot(int i) {
  std::lock_guard<std::mutex> lock(g_slot_mutex);
  if (i >= 0 && i < kConstSlots) g_slot_used[i] = false;
}

int drg_ctx_create(int device, drg_ctx** out) {
  if (!out) return DRG_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return DRG_ERR_NODEVICE;
  if (device < 0 || device >= count) return DRG_ERR_INVALID;
  drg_ctx* c = new (std::nothrow) drg_ctx();
  if (!c) return DRG_ERR_OOM;
  c->device = device;
  c->slot = acquire_slot();
  if (c->slot < 0) {
    delete c;
    return DRG_ERR_INVALID;  // more live contexts than constant banks
  }
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  const uint64_t keep = UINT64_MAX;  // hold freed blocks for reuse by the next call
  int prio_low = 0, prio_high = 0;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess ||
      // the side stream carries the long warps of the score pass: its blocks
      // are dispatched ahead of the bulk class's whenever an SM frees up
      cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
      cudaMemPoolCreate(&c->pool, &props) != cudaSuccess ||
      cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, (void*)&keep) != cudaSuccess) {
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->pool) cudaMemPoolDestroy(c->pool);
    release_slot(c->slot);
    delete c;
    return DRG_ERR_CUDA;
  }
  // the radix sort's error word starts clear: a new allocation may hold a
  // freed buffer's bytes, which every later check would read as a timeout
  try {
    DRG_CUDA(cudaMemsetAsync(c->sort_err.as<uint32_t>(1), 0, sizeof(uint32_t), c->stream));
    DRG_CUDA(cudaStreamSynchronize(c->stream));
  } catch (const Error& e) {
    drg_ctx_destroy(c);
    return e.code;
  }
  *out = c;
  return DRG_OK;
}

void drg_ctx_destroy(drg_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaStreamSynchronize(c->side);
  cudaStreamDestroy(c->stream);
  cudaStreamDestroy(c->side);
  cudaMemPoolDestroy(c->pool);  // released once the last resident buffer is freed
  release_slot(c->slot);
  delete c;
}

const char* drg_last_error(const drg_ctx* c) { return c ? c->err.c_str() : "no context"; }

int drg_ctx_get_tuning(const drg_ctx* c, drg_tuning* out) {
  if (!c || !out) return DRG_ERR_INVALID;
  *out = c->tuning;
  return DRG_OK;
}

int drg_ctx_set_tuning(drg_ctx* c, const drg_tuning* t) {
  if (!c || !t) return DRG_ERR_INVALID;
  const int w = t->sw_wide_min_width, p = t->sw_min_packed_width;
  if ((w != 137 && w != 273 && w != 545 && w != 1701) || (p != 17 && p != 33) ||
      (t->sw_transpose != 0 && t->sw_transpose != 1) || (t->sort_small_tiles != 0 && t->sort_small_tiles != 1)) {
    c->err = "tuning value outside its list (include/drgpu.h)";
    return DRG_ERR_INVALID;
  }
  c->tuning = *t;
  return DRG_OK;
}

int drg_seed_chunks(uint64_t n, uint64_t parts, uint64_t* out_pairs, uint64_t* n_out) {
  if (!n_out) return DRG_ERR_INVALID;
  auto v = split_chunks(n, parts);
  for (size_t i = 0; i < v.size(); ++i) {
    if (out_pairs) {
      out_pairs[2 * i] = v[i].first;
      out_pairs[2 * i + 1] = v[i].second;
    }
  }
  *n_out = v.size();
  return DRG_OK;
}

int drg_radix_sort(drg_ctx* c, void* keys, int32_t key_bytes, uint32_t* vals, uint64_t n, int32_t begin_bit,
                   int32_t end_bit, int32_t count_on_device) {
  if (!c || (n && !keys) || (key_bytes != 4 && key_bytes != 8) || begin_bit < 0 || end_bit < begin_bit ||
      end_bit > 8 * key_bytes)
    return DRG_ERR_INVALID;
  API_BEGIN(c)
  if (n >= (1ull << 32)) throw Error(DRG_ERR_INVALID, "radix sort: at most 2^32 - 1 keys");
  // with the count on the device, the buffers hold a larger capacity (tiles
  // past the count are never taken), as when a sort follows the kernel that
  // counted its input
  const uint64_t cap = count_on_device ? 2 * n + 5000 : n;
  DevArr<uint8_t> k(cap * key_bytes), ka(cap * key_bytes);
  DevArr<uint32_t> v(vals ? cap : 0), va(vals ? cap : 0);
  DevArr<uint64_t> dn(1);
  if (n) DRG_CUDA(cudaMemcpyAsync(k.p, keys, n * key_bytes, cudaMemcpyHostToDevice, c->stream));
  if (n && vals) DRG_CUDA(cudaMemcpyAsync(v.p, vals, n * 4, cudaMemcpyHostToDevice, c->stream));
  DRG_CUDA(cudaMemcpyAsync(dn.p, &n, sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
  const uint64_t* d_n = count_on_device ? dn.p : nullptr;
  void* rk;
  uint32_t* rv;
  if (key_bytes == 4) {
    auto r = radix_sort<uint32_t>(reinterpret_cast<uint32_t*>(k.p), reinterpret_cast<uint32_t*>(ka.p),
                                  vals ? v.p : nullptr, vals ? va.p : nullptr, cap, d_n, begin_bit, end_bit,
                                  c->sort_tmp, c->sort_err.as<uint32_t>(1), c->stream);
    rk = r.keys;
    rv = r.vals;
  } else {
    auto r = radix_sort<uint64_t>(reinterpret_cast<uint64_t*>(k.p), reinterpret_cast<uint64_t*>(ka.p),
                                  vals ? v.p : nullptr, vals ? va.p : nullptr, cap, d_n, begin_bit, end_bit,
                                  c->sort_tmp, c->sort_err.as<uint32_t>(1), c->stream);
    rk = r.keys;
    rv = r.vals;
  }
  if (n) DRG_CUDA(cudaMemcpyAsync(keys, rk, n * key_bytes, cudaMemcpyDeviceToHost, c->stream));
  if (n && vals) DRG_CUDA(cudaMemcpyAsync(vals, rv, n * 4, cudaMemcpyDeviceToHost, c->stream));
  sync(c);
  API_END(c)
}

int drg_seed_build(drg_ctx* c, const uint8_t* letters, const uint64_t* offsets, uint64_t n_seqs,
                   const char* shape_code, int32_t reduction, uint32_t base, double complexity_cut,
                   drg_seed_entry** out, uint64_t* n_out) {
  if (!c || !offsets || !shape_code || !out || !n_out) return DRG_ERR_INVALID;
  API_BEGIN(c)
  ShapeCode sh;
  if (!parse_shape(shape_code, &sh))
    throw Error(DRG_ERR_INVALID, std::string("invalid seed shape \"") + shape_code + "\": expected only 0/1");
  if (sh.weight > kMaxWeight) throw Error(DRG_ERR_INVALID, "seed shape weight above 16");
  if (sh.span > kMaxSpan) throw Error(DRG_ERR_INVALID, "seed shape longer than 256 positions");
  if (reduction < 0 || reduction > 2) throw Error(DRG_ERR_INVALID, "unknown reduction id");
  ReducedAlphabet red = reduction_by_id(reduction);
  ShapeTable t{};
  t.n = 1;
  t.weight[0] = (uint8_t)sh.weight;
  t.span[0] = (uint16_t)sh.span;
  for (int k = 0; k < sh.weight; ++k) t.pos[0][k] = (uint8_t)sh.positions[k];
  SeedParams p{};
  for (int i = 0; i < 32; ++i) p.bucket[i] = 255;
  for (int i = 0; i < 25; ++i) p.bucket[i] = red.bucket[i];
  p.size = (uint64_t)red.size;
  p.cut = complexity_cut;
  ln_factorial_table(p.lnfact);
  p.shape_shift = 48;  // one shape: the key is the shape's packed key
  p.request_shift = 56;
  Seqs s;
  s.upload(c, letters, offsets, n_seqs);
  upload_seed_params(t, p, c->slot, c->stream);
  const uint64_t N = s.total;
  DevArr<uint64_t> k(N), ks(N);
  DevArr<uint32_t> v(N), vs(N);
  launch_seed_enum(s.letters, s.offsets, s.owner, 0, s.total, 1, k.p, v.p, c->slot, c->stream);
  const SortResult<uint64_t> sr = radix_sort<uint64_t>(k.p, ks.p, v.p, vs.p, N, nullptr, 0, 64, c->sort_tmp,
                                                       c->sort_err.as<uint32_t>(1), c->stream);
  std::vector<uint64_t> hk(N);
  std::vector<uint32_t> hv(N);
  if (N) {
    DRG_CUDA(cudaMemcpyAsync(hk.data(), sr.keys, N * 8, cudaMemcpyDeviceToHost, c->stream));
    DRG_CUDA(cudaMemcpyAsync(hv.data(), sr.vals, N * 4, cudaMemcpyDeviceToHost, c->stream));
  }
  sync(c);
  uint64_t nv = 0;
  while (nv < N && hk[nv] != kNoSeed) ++nv;
  drg_seed_entry* o = (drg_seed_entry*)std::malloc(sizeof(drg_seed_entry) * (nv + 1));
  if (!o) throw Error(DRG_ERR_OOM, "host allocation failed");
  for (uint64_t i = 0; i < nv; ++i) {
    uint64_t g = hv[i];
    uint64_t seq = (uint64_t)(std::upper_bound(s.h_offsets.begin(), s.h_offsets.end(), g) - s.h_offsets.begin()) - 1;
    while (seq + 1 < s.h_offsets.size() && s.h_offsets[seq + 1] <= g) ++seq;  // empty sequences
    o[i].key = hk[i];
    o[i].seq = base + (uint32_t)seq;
    o[i].pos = (uint32_t)(g - s.h_offsets[seq]);
  }
  *out = o;
  *n_out = nv;
  API_END(c)
}

int drg_seed_join(drg_ctx* c, const drg_seed_entry* q, uint64_t nq, const drg_seed_entry* r, uint64_t nr,
                  uint64_t n_targets, uint64_t max_expand, drg_seed_hit** out, uint64_t* n_out) {
  if (!c || !out || !n_out || (nq && !q) || (nr && !r)) return DRG_ERR_INVALID;
  API_BEGIN(c)
  *out = nullptr;
  *n_out = 0;
  for (uint64_t i = 0; i < nq; ++i)
    if (q[i].seq >= n_targets) throw Error(DRG_ERR_INVALID, "query entry sequence index out of range");
  std::vector<uint64_t> qk(nq), rk(nr);
  std::vector<uint32_t> qseq(nq), qpos(nq), rseq(nr), rpos(nr), qid(nq), rid(nr);
  for (uint64_t i = 0; i < nq; ++i) {
    qk[i] = q[i].key;
    qseq[i] = q[i].seq;
    qpos[i] = q[i].pos;
    qid[i] = (uint32_t)i;
  }
  for (uint64_t i = 0; i < nr; ++i) {
    rk[i] = r[i].key;
    rseq[i] = r[i].seq;
    rpos[i] = r[i].pos;
    rid[i] = (uint32_t)i;
  }
  DevArr<uint64_t> dqk(nq), drk(nr), ukeys(nq + 1);
  DevArr<uint32_t> dqseq(nq), dqpos(nq), drseq(nr), drpos(nr), dqid(nq), drid(nr), ucount(nq + 1), ustart(nq + 1),
      rlo(nq + 1), rcnt(nq + 1);
  DevArr<uint64_t> uhits(nq + 2), uoff(nq + 2);
  DevArr<int64_t> cnt(2);
  auto up = [&](void* d, const void* h, size_t bytes) {
    if (bytes) DRG_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, c->stream));
  };
  up(dqk.p, qk.data(), nq * 8);
  up(drk.p, rk.data(), nr * 8);
  up(dqseq.p, qseq.data(), nq * 4);
  up(dqpos.p, qpos.data(), nq * 4);
  up(drseq.p, rseq.data(), nr * 4);
  up(drpos.p, rpos.data(), nr * 4);
  up(dqid.p, qid.data(), nq * 4);
  up(drid.p, rid.data(), nr * 4);
  int64_t n_runs = 0;
  if (nq > 0) {
    cub_run(c, [&](void* tmp, size_t& b) {
      return cub::DeviceRunLengthEncode::Encode(tmp, b, dqk.p, ukeys.p, ucount.p, cnt.p, (int64_t)nq, c->stream);
    });
    DRG_CUDA(cudaMemcpyAsync(&n_runs, cnt.p, 8, cudaMemcpyDeviceToHost, c->stream));
    sync(c);
  }
  if (n_runs > 0) {
    cub_run(c, [&](void* tmp, size_t& b) {
      return cub::DeviceScan::ExclusiveSum(tmp, b, ucount.p, ustart.p, n_runs, c->stream);
    });
    launch_join_count(ukeys.p, ucount.p, (uint64_t)n_runs, drk.p, nr, max_expand, rlo.p, rcnt.p, uhits.p, ~0ull,
                      c->stream);
    DRG_CUDA(cudaMemsetAsync(uhits.p + n_runs, 0, 8, c->stream));
    cub_run(c, [&](void* tmp, size_t& b) {
      return cub::DeviceScan::ExclusiveSum(tmp, b, uhits.p, uoff.p, n_runs + 1, c->stream);
    });
    uint64_t n_hits = 0;
    DRG_CUDA(cudaMemcpyAsync(&n_hits, uoff.p + n_runs, 8, cudaMemcpyDeviceToHost, c->stream));
    sync(c);
    DevArr<uint32_t> h4(4 * n_hits);
    JoinExpandArgs a{};
    a.run_hit_off = uoff.p;
    a.run_qstart = ustart.p;
    a.run_rlo = rlo.p;
    a.run_rcount = rcnt.p;
    a.n_runs = (uint64_t)n_runs;
    a.q_vals = dqid.p;
    a.r_vals = drid.p;
    a.n_hits = n_hits;
    a.q_seq = dqseq.p;
    a.q_pos = dqpos.p;
    a.r_seq = drseq.p;
    a.r_pos = drpos.p;
    a.hits4 = h4.p;
    launch_join_expand(a, c->stream);
    drg_seed_hit* o = (drg_seed_hit*)std::malloc(sizeof(drg_seed_hit) * (n_hits + 1));
    if (!o) throw Error(DRG_ERR_OOM, "host allocation failed");
    if (n_hits) DRG_CUDA(cudaMemcpyAsync(o, h4.p, n_hits * 16, cudaMemcpyDeviceToHost, c->stream));
    sync(c);
    std::sort(o, o + n_hits, [](const drg_seed_hit& x, const drg_seed_hit& y) {
      if (x.query != y.query) return x.query < y.query;
      if (x.subject != y.subject) return x.subject < y.subject;
      int64_t dx = (int64_t)x.qpos - x.spos, dy = (int64_t)y.qpos - y.spos;
      if (dx != dy) return dx < dy;
      return x.spos < y.spos;
    });
    *out = o;
    *n_out = n_hits;
  } else {
    *out = (drg_seed_hit*)std::malloc(sizeof(drg_seed_hit));
  }
  API_END(c)
}

int drg_xdrop_batch(drg_ctx* c, const uint8_t* ql, const uint64_t* qo, uint64_t nq, const uint8_t* sl,
                    const uint64_t* so, uint64_t ns, const drg_xdrop_job* jobs, uint64_t n, const char* matrix,
                    int32_t xdrop, drg_segment* out) {
  if (!c || !qo || !so || (n && (!jobs || !out))) return DRG_ERR_INVALID;
  API_BEGIN(c)
  Scoring sc;
  std::string err;
  if (!make_scoring(matrix, -1, -1, &sc, &err)) throw Error(DRG_ERR_INVALID, err);
  for (uint64_t i = 0; i < n; ++i) {
    if (jobs[i].query >= nq || jobs[i].subject >= ns) throw Error(DRG_ERR_INVALID, "job sequence index out of range");
    if (jobs[i].qa > qo[jobs[i].query + 1] - qo[jobs[i].query] || jobs[i].sa > so[jobs[i].subject + 1] - so[jobs[i].subject])
      throw Error(DRG_ERR_INVALID, "anchor outside its sequence");
  }
  Seqs qs, ss;
  qs.upload(c, ql, qo, nq);
  ss.upload(c, sl, so, ns);
  upload_score_matrix(sc.scores, c->slot, c->stream);
  DevArr<drg_xdrop_job> dj(n);
  DevArr<drg_segment> dout(n);
  if (n) DRG_CUDA(cudaMemcpyAsync(dj.p, jobs, n * sizeof(drg_xdrop_job), cudaMemcpyHostToDevice, c->stream));
  launch_xdrop_jobs(dj.p, n, qs.letters, qs.offsets, ss.letters, ss.offsets, xdrop, dout.p, c->slot, c->stream);
  if (n) DRG_CUDA(cudaMemcpyAsync(out, dout.p, n * sizeof(drg_segment), cudaMemcpyDeviceToHost, c->stream));
  sync(c);
  API_END(c)
}

int drg_extend_span_batch(drg_ctx* c, const uint8_t* ql, const uint64_t* qo, uint64_t nq, const uint8_t* sl,
                          const uint64_t* so, uint64_t ns, const drg_span_job* jobs, uint64_t n, const char* matrix,
                          int32_t go, int32_t ge, drg_aligned* out, uint32_t** ops, uint64_t* n_ops) {
  if (!c || !qo || !so || !ops || !n_ops || (n && (!jobs || !out))) return DRG_ERR_INVALID;
  API_BEGIN(c)
  Scoring sc;
  std::string err;
  if (!make_scoring(matrix, go, ge, &sc, &err)) throw Error(DRG_ERR_INVALID, err);
  Seqs qs, ss;
  qs.upload(c, ql, qo, nq);
  ss.upload(c, sl, so, ns);
  // one Band per job (whole query as the window); the band kernels take what
  // they support and the exact kernel the rest, as in the search's traceback
  std::vector<Band> hb(n);
  std::vector<uint64_t> ops_off(n + 1, 0);
  for (uint64_t i = 0; i < n; ++i) {
    const drg_span_job& j = jobs[i];
    if (j.query >= nq || j.subject >= ns) throw Error(DRG_ERR_INVALID, "job sequence index out of range");
    int64_t d0 = std::min(j.d0, j.d1), d1 = std::max(j.d0, j.d1);
    if (d0 < INT32_MIN / 2 || d1 > INT32_MAX / 2) throw Error(DRG_ERR_INVALID, "diagonal out of range");
    Band& b = hb[i];
    std::memset(&b, 0, sizeof b);
    b.target = j.query;
    b.subject = j.subject;
    b.d0 = (int32_t)d0;
    b.d1 = (int32_t)d1;
    b.n = (uint32_t)(qo[j.query + 1] - qo[j.query]);
    ops_off[i + 1] = ops_off[i] + b.n + (so[j.subject + 1] - so[j.subject]);
  }
  const uint64_t ooff = ops_off[n];
  DevArr<Band> db_(n);
  DevArr<ExactOut> dout(n);
  DevArr<uint32_t> dops(ooff + 1);
  DevArr<uint64_t> doff(n + 1);
  DevArr<int64_t> cnt(2);
  DevArr<unsigned long long> cells(4);  // evaluated, lane, issued cells, transposed bands
  DRG_CUDA(cudaMemsetAsync(cells.p, 0, 4 * sizeof(unsigned long long), c->stream));
  if (n) {
    DRG_CUDA(cudaMemcpyAsync(db_.p, hb.data(), n * sizeof(Band), cudaMemcpyHostToDevice, c->stream));
    DRG_CUDA(cudaMemsetAsync(dout.p, 0, n * sizeof(ExactOut), c->stream));
  }
  DRG_CUDA(cudaMemcpyAsync(doff.p, ops_off.data(), (n + 1) * 8, cudaMemcpyHostToDevice, c->stream));
  drg_run_stats st{};
  run_bands(c, db_.p, n, qs.view(), ss.view(), sc, true, nullptr, nullptr, dout.p, dops.p, doff.p, &ops_off, st,
            cnt.p, cells.p);
  std::vector<ExactOut> eo(n);
  std::vector<uint32_t> hops(ooff);
  if (n) DRG_CUDA(cudaMemcpyAsync(eo.data(), dout.p, n * sizeof(ExactOut), cudaMemcpyDeviceToHost, c->stream));
  if (ooff) DRG_CUDA(cudaMemcpyAsync(hops.data(), dops.p, ooff * 4, cudaMemcpyDeviceToHost, c->stream));
  sync(c);
  uint64_t total = 0;
  for (auto& e : eo) total += e.score > 0 ? e.n_ops : 0;
  uint32_t* o = (uint32_t*)std::malloc(sizeof(uint32_t) * (total + 1));
  if (!o) throw Error(DRG_ERR_OOM, "host allocation failed");
  uint64_t k = 0;
  for (uint64_t i = 0; i < n; ++i) {
    drg_aligned& a = out[i];
    std::memset(&a, 0, sizeof a);
    const Band& b = hb[i];
    a.cells = band_cells_host(b.n, (uint32_t)(so[b.subject + 1] - so[b.subject]), b.d0, b.d1);
    a.ops_offset = k;
    if (eo[i].score < 0) {
      std::free(o);
      throw Error(DRG_ERR_CUDA, "internal: traceback left the band");
    }
    if (eo[i].score == 0) continue;
    a.found = 1;
    a.score = eo[i].score;
    a.q_begin = eo[i].q_begin;
    a.q_end = eo[i].q_end;
    a.s_begin = eo[i].s_begin;
    a.s_end = eo[i].s_end;
    a.identities = eo[i].identities;
    a.positives = eo[i].positives;
    a.mismatches = eo[i].mismatches;
    a.gap_openings = eo[i].gap_openings;
    a.gaps = eo[i].gaps;
    a.length = eo[i].length;
    a.n_ops = eo[i].n_ops;
    std::memcpy(o + k, hops.data() + ops_off[i], eo[i].n_ops * 4);
    k += eo[i].n_ops;
  }
  *ops = o;
  *n_ops = k;
  API_END(c)
}

int drg_extend_span_scores(drg_ctx* c, const uint8_t* ql, const uint64_t* qo, uint64_t nq, const uint8_t* sl,
                           const uint64_t* so, uint64_t ns, const drg_span_job* jobs, uint64_t n, const char* matrix,
                           int32_t go, int32_t ge, int32_t* scores, drg_run_stats* stats) {
  if (!c || !qo || !so || (n && (!jobs || !scores))) return DRG_ERR_INVALID;
  API_BEGIN(c)
  Scoring sc;
  std::string err;
  if (!make_scoring(matrix, go, ge, &sc, &err)) throw Error(DRG_ERR_INVALID, err);
  Seqs qs, ss;
  qs.upload(c, ql, qo, nq);
  ss.upload(c, sl, so, ns);
  std::vector<Band> hb(n);
  for (uint64_t i = 0; i < n; ++i) {
    const drg_span_job& j = jobs[i];
    if (j.query >= nq || j.subject >= ns) throw Error(DRG_ERR_INVALID, "job sequence index out of range");
    int64_t d0 = std::min(j.d0, j.d1), d1 = std::max(j.d0, j.d1);
    if (d0 < INT32_MIN / 2 || d1 > INT32_MAX / 2) throw Error(DRG_ERR_INVALID, "diagonal out of range");
    Band& b = hb[i];
    std::memset(&b, 0, sizeof b);
    b.target = j.query;
    b.subject = j.subject;
    b.d0 = (int32_t)d0;
    b.d1 = (int32_t)d1;
    b.q0 = 0;
    b.n = (uint32_t)(qo[j.query + 1] - qo[j.query]);
  }
  DevArr<Band> db_(n);
  DevArr<int32_t> ds(n);
  DevArr<int64_t> cnt(2);
  DevArr<unsigned long long> cells(4);  // evaluated, lane, issued cells, transposed bands
  DRG_CUDA(cudaMemsetAsync(cells.p, 0, 4 * sizeof(unsigned long long), c->stream));
  if (n) DRG_CUDA(cudaMemcpyAsync(db_.p, hb.data(), n * sizeof(Band), cudaMemcpyHostToDevice, c->stream));
  drg_run_stats st{};
  run_bands(c, db_.p, n, qs.view(), ss.view(), sc, false, ds.p, nullptr, nullptr, nullptr, nullptr, nullptr, st, cnt.p,
            cells.p);
  if (n) DRG_CUDA(cudaMemcpyAsync(scores, ds.p, n * 4, cudaMemcpyDeviceToHost, c->stream));
  unsigned long long cg[4] = {0, 0, 0, 0};
  DRG_CUDA(cudaMemcpyAsync(cg, cells.p, sizeof(cg), cudaMemcpyDeviceToHost, c->stream));
  sync(c);
  st.dp_cells_gpu = cg[0];
  st.dp_cells_lane = cg[1];
  st.dp_cells_issued = cg[2];
  st.sw_transposed_bands = cg[3];
  if (stats) *stats = st;
  API_END(c)
}

int drg_db_create(drg_ctx* c, const uint8_t* letters, const uint64_t* offsets, uint64_t n, drg_db** out) {
  if (!c || !offsets || !out) return DRG_ERR_INVALID;
  API_BEGIN(c)
  *out = make_db(c, letters, offsets, n);
  API_END(c)
}

void drg_db_destroy(drg_db* d) {
  if (d) cudaSetDevice(d->ctx->device);
  free_db(d);
}

int drg_db_set_index_budget(drg_db* d, uint64_t budget_bytes) {
  if (!d || !d->cache) return DRG_ERR_INVALID;
  drg_ctx* c = d->ctx;
  API_BEGIN(c)
  d->cache->set_budget(budget_bytes);
  API_END(c)
}

int drg_db_index_stats(const drg_db* d, drg_index_stats* out) {
  if (!d || !d->cache || !out) return DRG_ERR_INVALID;
  const auto s = d->cache->stats();
  *out = drg_index_stats{s.entries, s.bytes, s.hits, s.misses, s.evictions};
  return DRG_OK;
}

int drg_batch_create(drg_ctx* c, const uint8_t* letters, const uint64_t* offsets, const uint32_t* query,
                     const uint8_t* frame, uint64_t n, drg_batch** out) {
  if (!c || !offsets || !out) return DRG_ERR_INVALID;
  API_BEGIN(c)
  *out = make_batch(c, letters, offsets, query, frame, n);
  API_END(c)
}

int drg_batch_create_requests(drg_ctx* c, const uint8_t* letters, const uint64_t* offsets, const uint32_t* query,
                              const uint8_t* frame, const uint32_t* request, uint64_t n, drg_batch** out) {
  if (!c || !offsets || !out || (n && !request)) return DRG_ERR_INVALID;
  API_BEGIN(c)
  *out = make_batch(c, letters, offsets, query, frame, n, request);
  API_END(c)
}

int drg_batch_create_blastx(drg_ctx* c, const uint8_t* nt, const uint64_t* nt_offsets, uint64_t n_reads,
                            int64_t min_orf, drg_batch** out) {
  if (!c || !nt_offsets || !out || (!nt && nt_offsets[n_reads] > 0)) return DRG_ERR_INVALID;
  API_BEGIN(c)
  *out = make_batch_translated(c, nt, nt_offsets, n_reads, min_orf);
  API_END(c)
}

int drg_translate_reads(drg_ctx* c, const uint8_t* nt, const uint64_t* nt_offsets, uint64_t n_reads,
                        int64_t min_orf, uint8_t** letters, uint64_t** offsets, uint32_t** query, uint8_t** frame,
                        uint64_t* n_targets) {
  if (!c || !nt_offsets || !letters || !offsets || !query || !frame || !n_targets ||
      (!nt && nt_offsets[n_reads] > 0))
    return DRG_ERR_INVALID;
  API_BEGIN(c)
  HostFrames h;
  drg_batch* b = make_batch_translated(c, nt, nt_offsets, n_reads, min_orf, &h);
  free_batch(b);
  const uint64_t n = h.query.size();
  *letters = (uint8_t*)std::malloc(h.letters.size() + 1);
  *offsets = (uint64_t*)std::malloc((n + 1) * sizeof(uint64_t));
  *query = (uint32_t*)std::malloc((n + 1) * sizeof(uint32_t));
  *frame = (uint8_t*)std::malloc(n + 1);
  if (!*letters || !*offsets || !*query || !*frame) {
    std::free(*letters);
    std::free(*offsets);
    std::free(*query);
    std::free(*frame);
    *letters = nullptr;
    *offsets = nullptr;
    *query = nullptr;
    *frame = nullptr;
    throw Error(DRG_ERR_OOM, "host allocation failed");
  }
  if (!h.letters.empty()) std::memcpy(*letters, h.letters.data(), h.letters.size());
  std::memcpy(*offsets, h.offsets.data(), (n + 1) * sizeof(uint64_t));
  if (n) std::memcpy(*query, h.query.data(), n * sizeof(uint32_t));
  if (n) std::memcpy(*frame, h.frame.data(), n);
  *n_targets = n;
  API_END(c)
}

int drg_batch_targets(const drg_batch* b, uint64_t* n_targets, uint32_t* query, uint8_t* frame) {
  if (!b || !n_targets) return DRG_ERR_INVALID;
  *n_targets = b->n;
  if (query && b->n) std::memcpy(query, b->query.data(), b->n * sizeof(uint32_t));
  if (frame && b->n) std::memcpy(frame, b->frame.data(), b->n);
  return DRG_OK;
}

void drg_batch_destroy(drg_batch* b) {
  if (b) cudaSetDevice(b->ctx->device);
  free_batch(b);
}

int drg_search_batch(drg_ctx* c, const drg_db* db, const drg_batch* b, const drg_search_config* cfg,
                     drg_result* out) {
  if (!c || !db || !b || !cfg || !out) return DRG_ERR_INVALID;
  std::memset(out, 0, sizeof *out);
  API_BEGIN(c)
  search(c, db, b, cfg, out);
  API_END(c)
}

int drg_search_run(drg_ctx* c, const uint8_t* dl, const uint64_t* dof, uint64_t ndb, const uint8_t* tl,
                   const uint64_t* tof, const uint32_t* tq, const uint8_t* tf, uint64_t nt,
                   const drg_search_config* cfg, drg_result* out) {
  if (!c || !dof || !tof || !cfg || !out) return DRG_ERR_INVALID;
  std::memset(out, 0, sizeof *out);
  API_BEGIN(c)
  auto t0 = std::chrono::steady_clock::now();
  drg_db* d = make_db(c, dl, dof, ndb);
  drg_batch* b = nullptr;
  try {
    b = make_batch(c, tl, tof, tq, tf, nt);
    double h2d = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    search(c, d, b, cfg, out);
    out->stats.ms_h2d = h2d;
  } catch (...) {
    free_batch(b);
    free_db(d);
    throw;
  }
  free_batch(b);
  free_db(d);
  API_END(c)
}

int drg_merge_frames(drg_result* res, uint64_t n_queries, const uint32_t* t_query, uint64_t max_hsps,
                     uint64_t max_targets) {
  if (!res || (res->n_targets && !t_query)) return DRG_ERR_INVALID;
  try {
    std::vector<std::vector<drg_hsp>> per(n_queries);
    for (uint64_t t = 0; t < res->n_targets; ++t) {
      uint32_t qi = t_query[t];
      if (qi >= n_queries) continue;
      for (uint64_t k = res->target_offsets[t]; k < res->target_offsets[t + 1]; ++k) per[qi].push_back(res->hsps[k]);
    }
    std::vector<drg_hsp> all;
    std::vector<uint64_t> offs(n_queries + 1, 0);
    std::vector<uint32_t> ops;
    for (uint64_t qi = 0; qi < n_queries; ++qi) {
      auto& v = per[qi];
      std::stable_sort(v.begin(), v.end(), [](const drg_hsp& a, const drg_hsp& b) { return cmp_hsp(a, b) < 0; });
      std::vector<uint32_t> order;
      std::unordered_map<uint32_t, std::vector<drg_hsp>> by;
      for (auto& h : v) {
        auto it = by.find(h.subject);
        if (it != by.end()) {
          if (it->second.size() < max_hsps) it->second.push_back(h);
        } else if (order.size() < max_targets) {
          order.push_back(h.subject);
          by[h.subject].push_back(h);
        }
      }
      for (uint32_t sid : order)
        for (auto h : by[sid]) {
          uint64_t o = ops.size();
          ops.insert(ops.end(), res->ops + h.ops_offset, res->ops + h.ops_offset + h.n_ops);
          h.ops_offset = o;
          all.push_back(h);
        }
      offs[qi + 1] = all.size();
    }
    std::free(res->hsps);
    std::free(res->target_offsets);
    std::free(res->ops);
    res->hsps = (drg_hsp*)std::malloc(sizeof(drg_hsp) * (all.size() + 1));
    res->target_offsets = (uint64_t*)std::malloc(sizeof(uint64_t) * (n_queries + 1));
    res->ops = (uint32_t*)std::malloc(sizeof(uint32_t) * (ops.size() + 1));
    if (!res->hsps || !res->target_offsets || !res->ops) return DRG_ERR_OOM;
    std::copy(all.begin(), all.end(), res->hsps);
    std::copy(offs.begin(), offs.end(), res->target_offsets);
    std::copy(ops.begin(), ops.end(), res->ops);
    res->n_hsps = all.size();
    res->n_targets = n_queries;
    res->n_ops = ops.size();
  } catch (const std::bad_alloc&) {
    return DRG_ERR_OOM;
  }
  return DRG_OK;
}

void drg_result_free(drg_result* r) {
  if (!r) return;
  std::free(r->hsps);
  std::free(r->target_offsets);
  std::free(r->ops);
  r->hsps = nullptr;
  r->target_offsets = nullptr;
  r->ops = nullptr;
  r->n_hsps = r->n_targets = r->n_ops = 0;
}

int drg_matrix_evalue(const char* matrix, int32_t go, int32_t ge, int32_t raw, uint64_t qlen, uint64_t slen,
                      uint64_t db_letters, double* evalue, double* bits) {
  Scoring sc;
  std::string err;
  if (!make_scoring(matrix, go, ge, &sc, &err)) return DRG_ERR_INVALID;
  if (evalue) *evalue = sc.evalue(raw, qlen, slen, db_letters);
  if (bits) *bits = sc.bit_score(raw);
  return DRG_OK;
}

int drg_probe_int_peak(drg_ctx* c, double* ops, double* mhz) {
  if (!c || !ops || !mhz) return DRG_ERR_INVALID;
  API_BEGIN(c)
  run_int_probe(ops, mhz, c->stream);
  API_END(c)
}

}  // extern "C"
