"""search::run parity on the GPU: every HSP field, bit for bit, against the
CPU oracle on seeded synthetic workloads, for every sensitivity preset."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import drgpu  # noqa: E402
from drgpu import synth  # noqa: E402


def as_tuples(lists):
    return [[h.key() for h in lst] for lst in lists]


def run_both(ctx, orc, w, **kw):
    dl, do = drgpu.concat(w.db)
    tl, to = drgpu.concat(w.queries)
    cfg = drgpu.make_config(**kw)
    got, stats = ctx.search(dl, do, tl, to, cfg)
    okw = dict(kw)
    exp, ostats = orc.search(w.db, w.queries, threads=8, **{k: v for k, v in okw.items()})
    return as_tuples(got), exp, stats, ostats


def small(config_id, n_queries, n_db, seed=0):
    return synth.workload(config_id, n_queries=n_queries, n_db=n_db, seed_offset=seed)


@pytest.mark.parametrize("sens", ["fast", "default", "mid-sensitive", "sensitive", "more-sensitive",
                                  "very-sensitive"])
def test_search_matches_oracle_all_presets(ctx, orc, sens):
    w = small(2, 24, 400, seed=1)
    got, exp, stats, ostats = run_both(ctx, orc, w, sensitivity=sens)
    assert got == exp
    assert stats["hits"] == ostats["hits"]
    assert sum(len(x) for x in exp) > 0


def test_search_ultra_sensitive(ctx, orc):
    w = small(2, 6, 150, seed=2)
    got, exp, _, _ = run_both(ctx, orc, w, sensitivity="ultra-sensitive")
    assert got == exp


@pytest.mark.parametrize("kw", [
    dict(sensitivity="sensitive", index_chunks=1),
    dict(sensitivity="sensitive", index_chunks=7),
    dict(sensitivity="default", max_hsps=3, max_target_seqs=4),
    dict(sensitivity="default", evalue=10.0),
    dict(sensitivity="sensitive", seed_cut=0.5),
    dict(sensitivity="default", matrix="BLOSUM80"),
    dict(sensitivity="default", matrix="PAM70", gap_open=10, gap_extend=1),
])
def test_search_options_match_oracle(ctx, orc, kw):
    w = small(2, 16, 300, seed=3)
    got, exp, _, _ = run_both(ctx, orc, w, **kw)
    assert got == exp


def test_search_config1_shape(ctx, orc):
    w = synth.workload(1, n_db=1200)
    got, exp, stats, _ = run_both(ctx, orc, w, sensitivity="default")
    assert got == exp
    assert len(exp[0]) >= 1


def test_search_empty_inputs(ctx):
    dl, do = drgpu.concat([np.zeros(10, np.uint8)])
    tl, to = drgpu.concat([])
    lists, _ = ctx.search(dl, do, tl, to, drgpu.make_config())
    assert lists == []
    tl, to = drgpu.concat([np.zeros(0, np.uint8), np.arange(20, dtype=np.uint8)])
    lists, _ = ctx.search(dl, do, tl, to, drgpu.make_config())
    assert len(lists) == 2 and lists[0] == []


def test_search_rejects_unknown_matrix(ctx):
    dl, do = drgpu.concat([np.zeros(10, np.uint8)])
    with pytest.raises(drgpu.DrgError) as ei:
        ctx.search(dl, do, dl, do, drgpu.make_config(matrix="NOPE"))
    assert ei.value.code == 1


def test_resident_search_equals_host_search(ctx):
    w = small(2, 12, 250, seed=4)
    dl, do = drgpu.concat(w.db)
    tl, to = drgpu.concat(w.queries)
    cfg = drgpu.make_config(sensitivity="sensitive")
    host, _ = ctx.search(dl, do, tl, to, cfg)
    db = drgpu.ResidentDb(ctx, dl, do)
    b = drgpu.ResidentBatch(ctx, tl, to)
    try:
        for _ in range(2):  # the resident objects can be searched repeatedly
            res, _, _ = drgpu.search_resident(ctx, db, b, cfg)
            assert as_tuples(res) == as_tuples(host)
    finally:
        b.close()
        db.close()


def test_search_with_letter_codes_above_24(ctx, orc):
    """Letter codes above 24 in the database and the queries: seeds skip them,
    scores treat them as 24, identities compare them as they are."""
    w = small(2, 20, 300, seed=9)
    r = np.random.Generator(np.random.PCG64(9))
    for seq in list(w.db) + list(w.queries):
        mask = r.random(len(seq)) < 0.03
        seq[mask] = r.choice(np.array([25, 31, 128, 255], np.uint8), size=int(mask.sum()))
    got, exp, _, _ = run_both(ctx, orc, w, sensitivity="sensitive")
    assert got == exp
    assert sum(len(x) for x in exp) > 0


def clip_workload():
    """One 5,000-aa query whose single subject holds 30 copies of 20-aa query
    pieces on diagonals 110 apart (-1650 .. +1540).  Each copy is an X-drop
    segment; their +-64 windows (band_for(5000) = 64, gapped.rs:27-32) overlap,
    so they merge into one band about 3,320 diagonals wide (search.rs:206-230).
    Then max_rows = max(16e6 / width, 2 * 64 + 16) ~ 4,800 < 5,000 and
    gapped_hsp clips the query rows around the anchor (search.rs:298-312)."""
    r = np.random.Generator(np.random.PCG64(7117))
    q = synth.random_protein(r, 5000)
    s = synth.random_protein(r, 5000)
    for k in range(30):
        qk = 100 + 150 * k
        d = -1650 + 110 * k
        sk = qk - d
        s[sk:sk + 20] = q[qk:qk + 20]
    db = [synth.random_protein(r, int(x)) for x in r.integers(100, 600, 40)]
    db.insert(17, s)
    return q, db


def test_search_window_clip(ctx, orc):
    q, db = clip_workload()
    dl, do = drgpu.concat(db)
    tl, to = drgpu.concat([q])
    for sens in ("default", "sensitive"):
        got, _ = ctx.search(dl, do, tl, to, drgpu.make_config(sensitivity=sens))
        exp, ostats = orc.search(db, [q], sensitivity=sens, threads=8)
        assert ostats["clipped_windows"] > 0
        assert as_tuples(got) == exp
        assert any(h[1] == 17 for h in exp[0])


def wide_key_workload():
    """1,100 queries against 1,500 subjects plus one of 4.2M aa holding 40 of
    the queries: the hit key (target | subject | diagonal | position) needs
    11 + 11 + 23 + 23 = 68 bits, so the search joins in windows of 128
    targets (7 bits) while every cap and HSP stays that of the whole batch."""
    r = np.random.Generator(np.random.PCG64(6464))
    queries = [synth.random_protein(r, int(x)) for x in r.integers(60, 160, 1100)]
    db = [synth.random_protein(r, int(x)) for x in r.integers(80, 300, 1500)]
    for j in range(0, 1500, 7):
        db[j] = synth.planted_homolog(r, queries[(j * 3) % 1100], 40, 100, 0.5, 0.7, 300)
    big = synth.random_protein(r, 4_200_000)
    for k in range(40):
        q = queries[k * 25]
        p = 50_000 + 100_000 * k
        big[p:p + len(q)] = q
    db.insert(500, big)
    return queries, db


def test_search_wide_hit_key_in_target_windows(ctx, orc):
    queries, db = wide_key_workload()
    dl, do = drgpu.concat(db)
    tl, to = drgpu.concat(queries)
    got, st = ctx.search(dl, do, tl, to, drgpu.make_config(sensitivity="default"))
    exp, _ = orc.search(db, queries, sensitivity="default", threads=8)
    assert st["query_blocks"] >= 9  # 1,100 targets in windows of 128, per index chunk
    assert as_tuples(got) == exp
    assert sum(1 for lst in exp for h in lst if h[1] == 500) == 40


def cap_workload():
    """60 queries and 80 database sequences that all hold one 24-aa motif, plus
    10 planted homologs.  With one index chunk every motif seed key has 60
    query and 80 reference occurrences: 4,800 > 4,096, so the reference's join
    drops those pairs (seed.rs:120-127, cap from search.rs:131).  Any 51
    queries alone stay under the cap, so a join that counted query
    occurrences per block instead of over the batch would report them."""
    r = np.random.Generator(np.random.PCG64(4242))
    motif = synth.random_protein(r, 24)
    queries = []
    for i in range(60):
        q = synth.random_protein(r, int(r.integers(200, 400)))
        p = int(r.integers(0, len(q) - 24))
        q[p:p + 24] = motif
        queries.append(q)
    db = []
    for j in range(80):
        s = synth.random_protein(r, int(r.integers(150, 500)))
        p = int(r.integers(0, len(s) - 24))
        s[p:p + 24] = motif
        db.append(s)
    for j in range(10):
        db.append(synth.planted_homolog(r, queries[j * 6], 120, 200, 0.5, 0.7, 400))
    return queries, db


@pytest.mark.parametrize("sens", ["default", "sensitive"])
def test_query_blocks_keep_the_batch_wide_cap(ctx, orc, sens):
    queries, db = cap_workload()
    dl, do = drgpu.concat(db)
    tl, to = drgpu.concat(queries)
    whole, wst = ctx.search(dl, do, tl, to, drgpu.make_config(sensitivity=sens, index_chunks=1))
    # a hit budget far below the batch's hits: the join runs in target blocks
    budget = max(200, wst["hits"] // 6)
    blocked, bst = ctx.search(dl, do, tl, to, drgpu.make_config(sensitivity=sens, index_chunks=1,
                                                                 max_hits_per_pass=budget))
    assert wst["query_blocks"] == 1
    assert bst["query_blocks"] >= 4 and bst["hit_passes"] >= 4
    assert bst["hits"] == wst["hits"]
    exp, _ = orc.search(db, queries, sensitivity=sens, index_chunks=1, threads=8)
    assert as_tuples(whole) == exp
    assert as_tuples(blocked) == exp
    # the construction crosses the cap: the first queries alone differ
    alone, _ = orc.search(db, queries[:20], sensitivity=sens, index_chunks=1, threads=8)
    assert alone != exp[:20]


def test_query_blocks_with_index_chunks(ctx, orc):
    w = small(2, 40, 600, seed=9)
    dl, do = drgpu.concat(w.db)
    tl, to = drgpu.concat(w.queries)
    exp, _ = orc.search(w.db, w.queries, sensitivity="sensitive", index_chunks=3, threads=8)
    got, st = ctx.search(dl, do, tl, to, drgpu.make_config(sensitivity="sensitive", index_chunks=3,
                                                            max_hits_per_pass=3000))
    assert st["query_blocks"] > 3
    assert as_tuples(got) == exp


@pytest.mark.parametrize("sens", ["fast", "default", "sensitive", "very-sensitive"])
def test_per_stage_drop_in_matches_oracle(ctx, orc, sens):
    """search::run orchestrated on the host over the stage entry points
    (drg_search_run_per_stage) equals the oracle and the fused search."""
    w = small(2, 24, 400, seed=1)
    dl, do = drgpu.concat(w.db)
    tl, to = drgpu.concat(w.queries)
    cfg = drgpu.make_config(sensitivity=sens, index_chunks=2)
    got, st, _ = ctx.search_per_stage(dl, do, tl, to, cfg)
    fused, _ = ctx.search(dl, do, tl, to, cfg)
    exp, ost = orc.search(w.db, w.queries, sensitivity=sens, index_chunks=2, threads=8)
    assert as_tuples(got) == exp
    assert as_tuples(fused) == exp
    assert st["hits"] == ost["hits"]
    assert sum(len(x) for x in exp) > 0


def test_per_stage_window_clip_and_cap(ctx, orc):
    q, db = clip_workload()
    dl, do = drgpu.concat(db)
    tl, to = drgpu.concat([q])
    got, _, _ = ctx.search_per_stage(dl, do, tl, to, drgpu.make_config(sensitivity="sensitive"))
    exp, _ = orc.search(db, [q], sensitivity="sensitive", threads=8)
    assert as_tuples(got) == exp
    queries, db = cap_workload()
    dl, do = drgpu.concat(db)
    tl, to = drgpu.concat(queries)
    got, _, _ = ctx.search_per_stage(dl, do, tl, to, drgpu.make_config(sensitivity="default", index_chunks=1))
    exp, _ = orc.search(db, queries, sensitivity="default", index_chunks=1, threads=8)
    assert as_tuples(got) == exp


@pytest.mark.parametrize("tuning", [dict(sw_wide_min_width=137), dict(sw_wide_min_width=545),
                                    dict(sw_wide_min_width=1701, sw_transpose=0),
                                    dict(sw_min_packed_width=33, sort_small_tiles=1)])
def test_tunings_give_identical_results(orc, tuning):
    """Every tile and routing choice of the autotuner gives the oracle's HSPs."""
    w = small(2, 24, 400, seed=3)
    dl, do = drgpu.concat(w.db)
    tl, to = drgpu.concat(w.queries)
    c = drgpu.Context(0)
    try:
        c.set_tuning(**tuning)
        assert all(c.tuning()[k] == v for k, v in tuning.items())
        for sens in ("sensitive", "very-sensitive"):
            got, _ = c.search(dl, do, tl, to, drgpu.make_config(sensitivity=sens))
            exp, _ = orc.search(w.db, w.queries, sensitivity=sens, threads=8)
            assert as_tuples(got) == exp
    finally:
        c.close()


def test_autotune_picks_and_caches(tmp_path):
    w = small(2, 60, 800, seed=4)
    dl, do = drgpu.concat(w.db)
    tl, to = drgpu.concat(w.queries)
    c = drgpu.Context(0)
    try:
        db = drgpu.ResidentDb(c, dl, do)
        b = drgpu.ResidentBatch(c, tl, to)
        cfg = drgpu.make_config(sensitivity="sensitive")
        cache = str(tmp_path / "tune.txt")
        t1, ms0, ms1 = c.autotune(db, b, cfg, cache_path=cache, reps=1)
        assert ms0 > 0 and 0 < ms1 <= ms0
        assert c.tuning() == t1
        c.set_tuning(sw_wide_min_width=1701)
        t2, a, _ = c.autotune(db, b, cfg, cache_path=cache, reps=1)  # answered by the cache
        assert t2 == t1 and a == 0 and c.tuning() == t1
        with pytest.raises(drgpu.DrgError):
            c.set_tuning(sw_wide_min_width=300)
        b.close()
        db.close()
    finally:
        c.close()


def test_long_extensions_run_by_the_warp(ctx, orc):
    """Subjects holding exact or lightly mutated copies of 600-1500-aa queries:
    their X-drop extensions run hundreds of cells, past the per-lane limit of
    128, so the warp finishes them (k_xdrop_runs); results must equal the
    oracle's."""
    r = np.random.Generator(np.random.PCG64(8181))
    queries = [synth.random_protein(r, int(n)) for n in r.integers(600, 1500, 12)]
    db = [synth.random_protein(r, int(n)) for n in r.integers(100, 800, 60)]
    for k, q in enumerate(queries):
        s = q.copy() if k % 2 == 0 else synth.mutate(r, q, 0.9, indel_rate=0.0)
        db[5 * k] = np.concatenate([synth.random_protein(r, 40), s, synth.random_protein(r, 30)])
    dl, do = drgpu.concat(db)
    tl, to = drgpu.concat(queries)
    for sens in ("fast", "sensitive"):
        got, _ = ctx.search(dl, do, tl, to, drgpu.make_config(sensitivity=sens))
        exp, _ = orc.search(db, queries, sensitivity=sens, threads=8)
        assert as_tuples(got) == exp
        assert sum(len(x) for x in exp) >= len(queries)
