"""Seed index cache of a resident database (GPU).

With a budget, the sorted reference seeds of each (preset, index chunk) stay
in device memory for later searches.  The cache must not change a single
result: every search below is compared with the same search on a database
without a cache, across presets, index chunks, evictions and two contexts
searching one database at once.
"""
import threading

import numpy as np
import pytest

import drgpu
from drgpu import synth

pytestmark = pytest.mark.gpu


def keys(lists):
    return [[h.key() for h in lst] for lst in lists]


@pytest.fixture(scope="module")
def case():
    w = synth.workload(2, n_queries=40, n_db=1500, seed_offset=41)
    dl, do = drgpu.concat(w.db)
    ql, qo = drgpu.concat(w.queries)
    return dl, do, ql, qo


def run(ctx, db, ql, qo, preset, chunks=1):
    b = drgpu.ResidentBatch(ctx, ql, qo)
    try:
        lists, st, _ = drgpu.search_resident(ctx, db, b, drgpu.make_config(sensitivity=preset, index_chunks=chunks))
    finally:
        b.close()
    return keys(lists), st


PRESETS = ["fast", "default", "sensitive", "very-sensitive"]
# Bytes a cached reference seed takes: a 4-byte letter index beside a 4-byte
# key when the sorted seed key (shape id included) fits 32 bits, else beside
# an 8-byte key.  Key bits per preset: fast 41, default 36, sensitive 32,
# very-sensitive 28.
SEED_BYTES = {"fast": 12, "default": 12, "sensitive": 8, "very-sensitive": 8}


def test_cached_index_gives_the_same_results(ctx, case):
    dl, do, ql, qo = case
    plain = drgpu.ResidentDb(ctx, dl, do)
    cached = drgpu.ResidentDb(ctx, dl, do, index_budget=1 << 34)
    try:
        held = 0
        for preset, chunks in [(p, 1) for p in PRESETS] + [("sensitive", 3)]:
            exp, st0 = run(ctx, plain, ql, qo, preset, chunks)
            assert st0["index_hits"] == 0
            first, st1 = run(ctx, cached, ql, qo, preset, chunks)   # builds the entries
            again, st2 = run(ctx, cached, ql, qo, preset, chunks)   # reads them
            assert first == exp and again == exp, preset
            assert st1["index_hits"] == 0 and st2["index_hits"] == chunks, preset
            assert st2["ref_seeds"] == st0["ref_seeds"] and st2["hits"] == st0["hits"]
            held += SEED_BYTES[preset] * st1["ref_seeds"]
        s = cached.index_stats()
        assert s["entries"] == len(PRESETS) + 3 and s["evictions"] == 0
        assert s["hits"] == len(PRESETS) + 3
        assert s["bytes"] == held and held > 0
        cached.set_index_budget(0)
        s = cached.index_stats()
        assert s["entries"] == 0 and s["bytes"] == 0
    finally:
        plain.close()
        cached.close()


def test_lru_eviction_under_a_small_budget(ctx, case):
    dl, do, ql, qo = case
    probe = drgpu.ResidentDb(ctx, dl, do, index_budget=1 << 34)
    plain = drgpu.ResidentDb(ctx, dl, do)
    try:
        run(ctx, probe, ql, qo, "fast")
        f = probe.index_stats()["bytes"]
        run(ctx, probe, ql, qo, "default")
        d = probe.index_stats()["bytes"] - f
        probe.close()
        probe = None
        # room for either preset's index, not for both
        budget = max(f, d) + min(f, d) // 2
        db = drgpu.ResidentDb(ctx, dl, do, index_budget=budget)
        try:
            expect = {p: run(ctx, plain, ql, qo, p)[0] for p in ("fast", "default")}
            for p in ("fast", "default", "fast", "default"):
                got, _ = run(ctx, db, ql, qo, p)
                assert got == expect[p], p
                assert db.index_stats()["entries"] == 1
            s = db.index_stats()
            assert s["bytes"] <= budget
            assert s["evictions"] == 3 and s["hits"] == 0
        finally:
            db.close()
    finally:
        if probe is not None:
            probe.close()
        plain.close()


def test_two_contexts_share_one_cache(ctx, case):
    dl, do, ql, qo = case
    plain = drgpu.ResidentDb(ctx, dl, do)
    expect = {p: run(ctx, plain, ql, qo, p)[0] for p in ("default", "sensitive")}
    plain.close()
    ctxs = [drgpu.Context(0) for _ in range(2)]
    db = drgpu.ResidentDb(ctxs[0], dl, do, index_budget=1 << 34)
    got, errors = {}, []

    def worker(k):
        try:
            for rep in range(3):
                p = ("default", "sensitive")[(k + rep) % 2]
                got[(k, rep)] = (p, run(ctxs[k], db, ql, qo, p)[0])
        except BaseException as e:  # re-raised below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    try:
        assert not errors, errors
        for (k, rep), (p, res) in got.items():
            assert res == expect[p], (k, rep, p)
        s = db.index_stats()
        # two threads may miss on one key together; both then build it once
        assert s["entries"] == 2 and s["hits"] + s["misses"] == 6 and s["hits"] >= 2
    finally:
        db.close()
        for c in ctxs:
            c.close()


def test_empty_database_with_a_budget(ctx):
    db = drgpu.ResidentDb(ctx, np.zeros(0, np.uint8), np.zeros(1, np.uint64), index_budget=1 << 20)
    try:
        ql, qo = drgpu.concat([synth.random_protein(np.random.Generator(np.random.PCG64(1)), 100)])
        lists, _ = run(ctx, db, ql, qo, "default")
        assert lists == [[]]
        assert db.index_stats()["entries"] == 0
    finally:
        db.close()
