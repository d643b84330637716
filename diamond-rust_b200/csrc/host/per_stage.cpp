// search::run (search.rs:95-146) and align_target (search.rs:148-271) as a
// caller of the per-stage entry points would write them: the reference's own
// orchestration on the host, each hot function replaced by its drop-in
// (drg_seed_build for seed::build, drg_seed_join for seed::join_into,
// drg_xdrop_batch for ungapped::xdrop, drg_extend_span_scores and
// drg_extend_span_batch for gapped::extend_span).  Every call takes host
// buffers and returns host results, as the crate's functions do.
//
// It is the plain form the fused search (drg_search_batch) is measured
// against, and a check that the stage entry points compose into search::run
// exactly.  Three steps are batched over all targets instead of being made
// per hit: every unique seed hit is X-dropped (the adjacency rule of
// search.rs:184-191 then picks the segments the reference would have
// extended: a skipped hit's extension is never used), every band's score is
// computed before the E-value walk, and the walk's survivors are traced in
// one call.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "drgpu.h"
#include "host/pool.h"
#include "host/presets.h"
#include "host/scoring.h"

namespace drg {
void set_context_error(drg_ctx* ctx, const std::string& msg);  // capi.cu
}

namespace {

using namespace drg;

constexpr double kLn2 = 0.693147180559945309417232121458176568;

struct Fail {
  int code;
};

void check(int rc) {
  if (rc != DRG_OK) throw Fail{rc};
}

// One seed hit of the join (seed.rs:21-27), ordered as align_target visits a
// subject's hits: by diagonal, then subject position (search.rs:178).
struct Hit {
  uint32_t target, subject, qpos, spos;
  int64_t diag() const { return (int64_t)qpos - (int64_t)spos; }
};
bool hit_less(const Hit& a, const Hit& b) {
  if (a.target != b.target) return a.target < b.target;
  if (a.subject != b.subject) return a.subject < b.subject;
  if (a.diag() != b.diag()) return a.diag() < b.diag();
  return a.spos < b.spos;
}
bool hit_same(const Hit& a, const Hit& b) {
  return a.target == b.target && a.subject == b.subject && a.qpos == b.qpos && a.spos == b.spos;
}

struct Seg {  // ungapped.rs:11-17
  uint64_t q_start, s_start, len;
  int32_t score;
  int64_t diag() const { return (int64_t)q_start - (int64_t)s_start; }
  uint64_t s_end() const { return s_start + len; }
};

// One band of a (target, subject) pair (search.rs:206-230) and its DP job.
struct BandJob {
  uint32_t target, subject;
  int64_t d0, d1;      // diagonals of the whole sequences
  uint64_t q0, q1;     // query window (search.rs:303-312)
  uint32_t query_seq;  // sequence the job's query is (a target, or a window slice)
  int32_t score = 0;
  double evalue = 0;
  bool kept = false;
};

struct Pair {
  uint32_t target, subject;
  uint64_t hit_lo, hit_hi;    // unique hits of the pair
  uint64_t band_lo, band_hi;  // its bands, in the order they get max_hsps
};

struct Found {  // one kept HSP
  uint32_t target, subject;
  uint64_t band;
  int32_t score;
  double evalue, bits;
  drg_aligned al;
  std::vector<uint32_t> ops;
};

int cmp_found(const Found& a, const Found& b) {  // cmp_hsp, search.rs:273-282
  if (a.score != b.score) return b.score < a.score ? -1 : 1;
  if (a.evalue < b.evalue) return -1;
  if (a.evalue > b.evalue) return 1;
  if (a.subject != b.subject) return a.subject < b.subject ? -1 : 1;
  return 0;
}

int reduction_id(const ReducedAlphabet& r) {
  for (int id = 0; id < 3; ++id) {
    const ReducedAlphabet x = reduction_by_id(id);
    if (x.size == r.size && std::memcmp(x.bucket, r.bucket, sizeof x.bucket) == 0) return id;
  }
  throw Fail{DRG_ERR_INVALID};
}

void run(drg_ctx* ctx, const uint8_t* db_letters, const uint64_t* db_offsets, uint64_t n_db, const uint8_t* t_letters,
         const uint64_t* t_offsets, const uint32_t* t_query, const uint8_t* t_frame, uint64_t n_targets,
         const drg_search_config* cfg, drg_result* out) {
  const auto t_start = std::chrono::steady_clock::now();
  std::memset(out, 0, sizeof(*out));
  Scoring sc;
  std::string err;
  const char* matrix = cfg->matrix ? cfg->matrix : "BLOSUM62";
  if (!make_scoring(matrix, cfg->gap_open, cfg->gap_extend, &sc, &err)) {
    set_context_error(ctx, err);
    throw Fail{DRG_ERR_INVALID};
  }
  const std::string sens = cfg->sensitivity ? cfg->sensitivity : "default";
  if (!known_sensitivity(sens)) {
    set_context_error(ctx, "unknown sensitivity " + sens);
    throw Fail{DRG_ERR_INVALID};
  }
  const std::vector<ShapeCode> shapes = preset_shapes(sens);
  const int red = reduction_id(preset_reduction(sens));
  const double cut = cfg->has_seed_cut ? cfg->seed_cut : preset_seed_cut(sens);
  const double complexity_cut = cut * kLn2 * (double)shapes[0].weight;  // search.rs:105
  const uint64_t chunks = cfg->index_chunks >= 0 ? std::max<int64_t>(cfg->index_chunks, 1)
                                                 : (uint64_t)preset_index_chunks(sens);
  const uint64_t max_hsps = std::max<uint32_t>(cfg->max_hsps, 1);
  const uint64_t max_targets = std::max<uint32_t>(cfg->max_target_seqs, 1);
  const int xdrop = sc.raw_score(12.3);  // search.rs:51-53
  const int cutoff = 19;                 // search.rs:164
  const uint64_t db_total = db_offsets[n_db];
  drg_run_stats st{};
  out->n_targets = n_targets;
  out->target_offsets = (uint64_t*)std::calloc(n_targets + 1, sizeof(uint64_t));
  if (!out->target_offsets) throw Fail{DRG_ERR_OOM};
  if (n_targets == 0 || n_db == 0) {
    out->hsps = (drg_hsp*)std::malloc(sizeof(drg_hsp));
    out->ops = (uint32_t*)std::malloc(sizeof(uint32_t));
    return;
  }
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  host::Pool pool(cfg->threads ? std::max(1u, cfg->threads) - 1 : std::min(hw - 1, 15u));

  // ---- seeds and join (search.rs:108-133)
  std::vector<drg_seed_entry*> qe(shapes.size(), nullptr);
  std::vector<uint64_t> nq(shapes.size(), 0);
  std::vector<Hit> hits;
  struct FreeSeeds {
    std::vector<drg_seed_entry*>* v;
    ~FreeSeeds() {
      for (auto* p : *v) drg_free(p);
    }
  } free_qe{&qe};
  for (size_t s = 0; s < shapes.size(); ++s) {
    check(drg_seed_build(ctx, t_letters, t_offsets, n_targets, shapes[s].code.c_str(), red, 0, complexity_cut, &qe[s],
                         &nq[s]));
    st.query_seeds += nq[s];
  }
  for (auto [c0, c1] : split_chunks(n_db, chunks)) {
    std::vector<uint64_t> off(c1 - c0 + 1);
    for (uint64_t i = c0; i <= c1; ++i) off[i - c0] = db_offsets[i] - db_offsets[c0];
    for (size_t s = 0; s < shapes.size(); ++s) {
      drg_seed_entry* re = nullptr;
      uint64_t nr = 0;
      check(drg_seed_build(ctx, db_letters + db_offsets[c0], off.data(), c1 - c0, shapes[s].code.c_str(), red,
                           (uint32_t)c0, complexity_cut, &re, &nr));
      st.ref_seeds += nr;
      drg_seed_hit* h = nullptr;
      uint64_t nh = 0;
      const int rc = drg_seed_join(ctx, qe[s], nq[s], re, nr, n_targets, 4096, &h, &nh);
      drg_free(re);
      check(rc);
      const size_t at = hits.size();
      hits.resize(at + nh);
      for (uint64_t k = 0; k < nh; ++k) hits[at + k] = Hit{h[k].query, h[k].subject, h[k].qpos, h[k].spos};
      drg_free(h);
    }
  }
  st.hits = hits.size();

  // ---- each target's hits by subject, diagonal, position (search.rs:172-178);
  // identical hits (from several shapes or chunks) extend to identical
  // segments, and the adjacency rule skips or re-scores the copies alike
  {
    std::vector<uint64_t> per(n_targets + 1, 0);
    for (const Hit& h : hits) ++per[h.target + 1];
    for (uint64_t t = 0; t < n_targets; ++t) per[t + 1] += per[t];
    std::vector<Hit> by(hits.size());
    std::vector<uint64_t> at(per.begin(), per.end() - 1);
    for (const Hit& h : hits) by[at[h.target]++] = h;
    hits.swap(by);
    pool.parallel_for(n_targets, 16, 0, [&](uint64_t lo, uint64_t hi) {
      for (uint64_t t = lo; t < hi; ++t) std::sort(hits.begin() + per[t], hits.begin() + per[t + 1], hit_less);
    });
    hits.erase(std::unique(hits.begin(), hits.end(), hit_same), hits.end());
  }
  st.unique_hits = hits.size();

  // ---- ungapped::xdrop of every unique hit (ungapped.rs:38-88)
  std::vector<drg_segment> segs(hits.size());
  {
    std::vector<drg_xdrop_job> jobs(hits.size());
    for (size_t i = 0; i < hits.size(); ++i)
      jobs[i] = drg_xdrop_job{hits[i].target, hits[i].subject, hits[i].qpos, hits[i].spos};
    check(drg_xdrop_batch(ctx, t_letters, t_offsets, n_targets, db_letters, db_offsets, n_db, jobs.data(),
                          jobs.size(), matrix, xdrop, segs.data()));
  }
  st.xdrops = hits.size();

  // ---- pairs, segments, bands and windows (search.rs:180-230, 298-312)
  std::vector<Pair> pairs;
  for (uint64_t i = 0; i < hits.size();) {
    uint64_t j = i;
    while (j < hits.size() && hits[j].target == hits[i].target && hits[j].subject == hits[i].subject) ++j;
    pairs.push_back(Pair{hits[i].target, hits[i].subject, i, j, 0, 0});
    i = j;
  }
  std::vector<std::vector<BandJob>> pair_bands(pairs.size());
  std::vector<uint64_t> pair_segments(pairs.size(), 0);
  pool.parallel_for(pairs.size(), 64, 0, [&](uint64_t lo, uint64_t hi) {
    std::vector<Seg> sg;
    std::vector<size_t> order;
    for (uint64_t p = lo; p < hi; ++p) {
      const Pair& pr = pairs[p];
      const uint64_t qlen = t_offsets[pr.target + 1] - t_offsets[pr.target];
      const uint64_t slen = db_offsets[pr.subject + 1] - db_offsets[pr.subject];
      if (qlen == 0 || slen == 0) continue;
      sg.clear();
      for (uint64_t k = pr.hit_lo; k < pr.hit_hi; ++k) {
        const Hit& h = hits[k];
        if (!sg.empty() && sg.back().diag() == h.diag() && sg.back().s_end() >= h.spos) continue;
        const drg_segment& x = segs[k];
        if (x.score >= cutoff) sg.push_back(Seg{x.q_start, x.s_start, x.len, x.score});
      }
      pair_segments[p] = sg.size();
      if (sg.empty()) continue;
      // by score, best first; ties keep the diagonal order (the reference's
      // unstable sort leaves them unspecified)
      std::stable_sort(sg.begin(), sg.end(), [](const Seg& a, const Seg& b) { return a.score > b.score; });
      const int64_t band = band_for_length(qlen);
      order.resize(sg.size());
      for (size_t k = 0; k < sg.size(); ++k) order[k] = k;
      std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return sg[a].diag() < sg[b].diag(); });
      struct B {
        int64_t d0, d1;
        size_t best;
      };
      std::vector<B> bs;
      for (size_t idx : order) {
        const int64_t d = sg[idx].diag(), b0 = d - band, b1 = d + band;
        if (!bs.empty() && b0 <= bs.back().d1) {
          bs.back().d1 = std::max(bs.back().d1, b1);
          if (sg[idx].score > sg[bs.back().best].score) bs.back().best = idx;
        } else {
          bs.push_back(B{b0, b1, idx});
        }
      }
      std::stable_sort(bs.begin(), bs.end(),
                       [&](const B& a, const B& b) { return sg[a.best].score > sg[b.best].score; });
      auto& out_b = pair_bands[p];
      for (const B& b : bs) {
        BandJob j;
        j.target = pr.target;
        j.subject = pr.subject;
        j.d0 = b.d0;
        j.d1 = b.d1;
        const uint64_t row_cells = (uint64_t)std::max<int64_t>(b.d1 - b.d0, 0) + 1;
        const uint64_t max_rows = std::max<uint64_t>(16000000ull / row_cells, 2 * (uint64_t)band + 16);
        uint64_t q0 = 0, q1 = qlen;
        if (q1 - q0 > max_rows) {
          const uint64_t anchor = sg[b.best].q_start;
          q0 = anchor >= max_rows / 2 ? anchor - max_rows / 2 : 0;
          q1 = std::min(q0 + max_rows, qlen);
          q0 = q1 >= max_rows ? q1 - max_rows : 0;
        }
        j.q0 = q0;
        j.q1 = q1;
        j.query_seq = pr.target;
        out_b.push_back(j);
      }
    }
  });
  std::vector<BandJob> bands;
  for (uint64_t p = 0; p < pairs.size(); ++p) {
    st.segments += pair_segments[p];
    pairs[p].band_lo = bands.size();
    for (auto& b : pair_bands[p]) bands.push_back(b);
    pairs[p].band_hi = bands.size();
    std::vector<BandJob>().swap(pair_bands[p]);
  }
  st.bands = bands.size();

  // windows clipped to fewer query rows are sequences of their own
  std::vector<uint8_t> wl;
  std::vector<uint64_t> wo;
  const uint8_t* ql = t_letters;
  const uint64_t* qo = t_offsets;
  uint64_t nqs = n_targets;
  {
    bool clipped = false;
    for (const auto& b : bands) clipped |= b.q0 != 0 || b.q1 != t_offsets[b.target + 1] - t_offsets[b.target];
    if (clipped) {
      wl.assign(t_letters, t_letters + t_offsets[n_targets]);
      wo.assign(t_offsets, t_offsets + n_targets + 1);
      for (auto& b : bands) {
        if (b.q0 == 0 && b.q1 == t_offsets[b.target + 1] - t_offsets[b.target]) continue;
        wl.insert(wl.end(), t_letters + t_offsets[b.target] + b.q0, t_letters + t_offsets[b.target] + b.q1);
        wo.push_back(wl.size());
        b.query_seq = (uint32_t)(wo.size() - 2);
      }
      ql = wl.data();
      qo = wo.data();
      nqs = wo.size() - 1;
    }
  }
  // window-local diagonals (search.rs:320-328)
  auto span_job = [&](const BandJob& b) {
    return drg_span_job{b.query_seq, b.subject, b.d0 - (int64_t)b.q0, b.d1 - (int64_t)b.q0};
  };

  // ---- scores of every band (gapped::extend_span, gapped.rs:67-203)
  {
    std::vector<drg_span_job> jobs(bands.size());
    for (size_t i = 0; i < bands.size(); ++i) jobs[i] = span_job(bands[i]);
    std::vector<int32_t> scores(bands.size(), 0);
    drg_run_stats sst{};
    check(drg_extend_span_scores(ctx, ql, qo, nqs, db_letters, db_offsets, n_db, jobs.data(), jobs.size(), matrix,
                                 sc.gap_open, sc.gap_extend, scores.data(), &sst));
    for (size_t i = 0; i < bands.size(); ++i) bands[i].score = scores[i];
    st.dp_cells_gpu = sst.dp_cells_gpu;
  }
  // ---- the E-value walk of each pair (search.rs:233-255), with E-values of
  // the full lengths (search.rs:335-338)
  pool.parallel_for(pairs.size(), 64, 0, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t p = lo; p < hi; ++p) {
      const Pair& pr = pairs[p];
      const uint64_t qlen = t_offsets[pr.target + 1] - t_offsets[pr.target];
      const uint64_t slen = db_offsets[pr.subject + 1] - db_offsets[pr.subject];
      uint64_t kept = 0;
      for (uint64_t k = pr.band_lo; k < pr.band_hi && kept < max_hsps; ++k) {
        BandJob& b = bands[k];
        if (b.score <= 0) continue;  // extend_span gave None
        b.evalue = sc.evalue(b.score, qlen, slen, db_total);
        if (b.evalue <= cfg->evalue) {
          b.kept = true;
          ++kept;
        }
      }
    }
  });
  // ---- traceback of the kept bands (gapped.rs:205-279)
  std::vector<uint64_t> kept;
  for (uint64_t k = 0; k < bands.size(); ++k)
    if (bands[k].kept) kept.push_back(k);
  std::vector<drg_aligned> al(kept.size());
  uint32_t* ops = nullptr;
  uint64_t n_ops = 0;
  {
    std::vector<drg_span_job> jobs(kept.size());
    for (size_t i = 0; i < kept.size(); ++i) jobs[i] = span_job(bands[kept[i]]);
    check(drg_extend_span_batch(ctx, ql, qo, nqs, db_letters, db_offsets, n_db, jobs.data(), jobs.size(), matrix,
                                sc.gap_open, sc.gap_extend, al.data(), &ops, &n_ops));
  }
  std::unique_ptr<uint32_t, void (*)(void*)> ops_owner(ops, drg_free);
  st.traced_bands = kept.size();

  // ---- per target: pairs in subject order, HSPs by cmp_hsp, targets by their
  // best HSP, --max-target-seqs, --max-hsps (search.rs:256-270)
  std::vector<std::vector<Found>> per_target(n_targets);
  for (size_t i = 0; i < kept.size(); ++i) {
    const BandJob& b = bands[kept[i]];
    const drg_aligned& a = al[i];
    if (!a.found || a.score != b.score) {
      set_context_error(ctx, "internal: traceback score differs from the band score");
      throw Fail{DRG_ERR_CUDA};
    }
    Found f;
    f.target = b.target;
    f.subject = b.subject;
    f.band = kept[i];
    f.score = a.score;
    f.evalue = b.evalue;
    f.bits = sc.bit_score(a.score);
    f.al = a;
    f.ops.assign(ops + a.ops_offset, ops + a.ops_offset + a.n_ops);
    per_target[b.target].push_back(std::move(f));
  }
  std::vector<std::vector<Found>> final_lists(n_targets);
  pool.parallel_for(n_targets, 16, 0, [&](uint64_t lo, uint64_t hi) {
    for (uint64_t t = lo; t < hi; ++t) {
      auto& v = per_target[t];  // already in subject order (pairs are)
      std::vector<std::vector<Found>> found;
      for (size_t i = 0; i < v.size();) {
        size_t j = i;
        while (j < v.size() && v[j].subject == v[i].subject) ++j;
        std::vector<Found> hs(std::make_move_iterator(v.begin() + i), std::make_move_iterator(v.begin() + j));
        std::stable_sort(hs.begin(), hs.end(), [](const Found& a, const Found& b) { return cmp_found(a, b) < 0; });
        found.push_back(std::move(hs));
        i = j;
      }
      std::stable_sort(found.begin(), found.end(), [](const std::vector<Found>& a, const std::vector<Found>& b) {
        return cmp_found(a[0], b[0]) < 0;
      });
      if (found.size() > max_targets) found.resize(max_targets);
      for (auto& hs : found) {
        if (hs.size() > max_hsps) hs.resize(max_hsps);
        for (auto& f : hs) final_lists[t].push_back(std::move(f));
      }
    }
  });
  uint64_t n_hsps = 0, total_ops = 0;
  for (const auto& l : final_lists) {
    n_hsps += l.size();
    for (const auto& f : l) total_ops += f.ops.size();
  }
  out->hsps = (drg_hsp*)std::malloc(sizeof(drg_hsp) * (n_hsps + 1));
  out->ops = (uint32_t*)std::malloc(sizeof(uint32_t) * (total_ops + 1));
  if (!out->hsps || !out->ops) throw Fail{DRG_ERR_OOM};
  uint64_t h = 0, ko = 0;
  for (uint64_t t = 0; t < n_targets; ++t) {
    for (const Found& f : final_lists[t]) {
      const BandJob& b = bands[f.band];
      drg_hsp& o = out->hsps[h++];
      o.query = t_query ? t_query[t] : (uint32_t)t;
      o.subject = f.subject;
      o.frame = t_frame ? t_frame[t] : 0;
      o.score = f.score;
      o.q_begin = (uint32_t)(b.q0 + f.al.q_begin);
      o.q_end = (uint32_t)(b.q0 + f.al.q_end);
      o.s_begin = (uint32_t)f.al.s_begin;
      o.s_end = (uint32_t)f.al.s_end;
      o.bits = f.bits;
      o.evalue = f.evalue;
      o.identities = f.al.identities;
      o.positives = f.al.positives;
      o.mismatches = f.al.mismatches;
      o.gap_openings = f.al.gap_openings;
      o.gaps = f.al.gaps;
      o.length = f.al.length;
      o.ops_offset = ko;
      o.n_ops = (uint32_t)f.ops.size();
      o.pad = 0;
      if (!f.ops.empty()) std::memcpy(out->ops + ko, f.ops.data(), f.ops.size() * sizeof(uint32_t));
      ko += f.ops.size();
    }
    out->target_offsets[t + 1] = h;
  }
  out->n_hsps = h;
  out->n_ops = ko;
  st.hsps = h;
  st.seed_shapes = shapes.size();
  st.ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  out->stats = st;
}

}  // namespace

extern "C" int drg_search_run_per_stage(drg_ctx* ctx, const uint8_t* db_letters, const uint64_t* db_offsets,
                                        uint64_t n_db, const uint8_t* t_letters, const uint64_t* t_offsets,
                                        const uint32_t* t_query, const uint8_t* t_frame, uint64_t n_targets,
                                        const drg_search_config* cfg, drg_result* out) {
  if (!ctx || !db_offsets || !t_offsets || !cfg || !out || (n_db && !db_letters) || (n_targets && !t_letters))
    return DRG_ERR_INVALID;
  try {
    run(ctx, db_letters, db_offsets, n_db, t_letters, t_offsets, t_query, t_frame, n_targets, cfg, out);
    return DRG_OK;
  } catch (const Fail& f) {
    drg_result_free(out);
    return f.code;
  } catch (const std::bad_alloc&) {
    drg_result_free(out);
    set_context_error(ctx, "host allocation failed");
    return DRG_ERR_OOM;
  }
}
