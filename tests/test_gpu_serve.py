"""Serving: requests batched together give the results they give alone (GPU).

The join cap (qcount x rcount <= 4096) counts a seed key's query occurrences
over the whole batch, so a plain mixed batch can change a request's hits.
drg_batch_create_requests counts them per request; these tests check every
request's HSP lists against its solo search (tolerance 0) and against the
oracle, and run a short request stream through the continuous-batching server.
"""
import numpy as np
import pytest

import drgpu
from drgpu import serve, synth

pytestmark = pytest.mark.gpu

MOTIF = "MKWVTFISLLHCDGQE"


def enc(text):
    return np.array([synth.AA.index(c) for c in text], np.uint8)


def cap_case():
    """A database where one motif occurs 100 times, and two requests of 30
    motif-carrying queries each: alone a request stays under the join cap for
    the motif's seeds (30 x 100), together it would not (60 x 100)."""
    rng = np.random.Generator(np.random.PCG64(77))
    db = synth.make_db(rng, 300, mean=200, lo=60, hi=400)
    for i in range(100):
        s = db[i].copy()
        at = int(rng.integers(0, len(s) - len(MOTIF)))
        s[at:at + len(MOTIF)] = enc(MOTIF)
        db[i] = s
    reqs = []
    for k in range(2):
        qs = []
        for _ in range(30):
            q = synth.random_protein(rng, int(rng.integers(80, 200)))
            at = int(rng.integers(0, len(q) - len(MOTIF)))
            q[at:at + len(MOTIF)] = enc(MOTIF)
            qs.append(q)
        qs += [synth.random_protein(rng, int(rng.integers(50, 300))) for _ in range(5)]
        reqs.append(serve.Request(k, "default", qs))
    return db, reqs


def keys(req):
    return [[h.key() for h in lst] for lst in req.results]


def solo(ctx, db, req, preset):
    r = serve.Request(req.rid, preset, req.queries)
    serve.search_batch(ctx, db, [r], preset)
    return keys(r)


def test_requests_mixed_equal_alone_across_the_join_cap(ctx, orc):
    db_seqs, reqs = cap_case()
    dl, do = drgpu.concat(db_seqs)
    db = drgpu.ResidentDb(ctx, dl, do)
    try:
        alone = [solo(ctx, db, r, "default") for r in reqs]
        serve.search_batch(ctx, db, reqs, "default")
        for r, a in zip(reqs, alone):
            assert keys(r) == a
        # the same queries as ONE request (the reference's batch semantics)
        # cross the cap: the per-request accounting is what keeps them apart
        merged = serve.Request(9, "default", reqs[0].queries + reqs[1].queries)
        serve.search_batch(ctx, db, [merged], "default")
        n0 = len(reqs[0].queries)
        shifted = [[(k[0] + n0,) + k[1:] for k in lst] for lst in alone[1]]
        assert keys(merged) != alone[0] + shifted
        # and each request alone is the reference path's answer
        for r, a in zip(reqs, alone):
            exp, _ = orc.search(db_seqs, r.queries, sensitivity="default", threads=8)
            assert a == exp
    finally:
        db.close()


@pytest.mark.parametrize("preset", ["fast", "sensitive", "very-sensitive", "ultra-sensitive"])
def test_mixed_batches_equal_alone(ctx, preset):
    w = synth.workload(2, n_queries=30, n_db=900, seed_offset=21)
    dl, do = drgpu.concat(w.db)
    db = drgpu.ResidentDb(ctx, dl, do)
    try:
        reqs = [serve.Request(k, preset, w.queries[k * 6:(k + 1) * 6]) for k in range(5)]
        alone = [solo(ctx, db, r, preset) for r in reqs]
        serve.search_batch(ctx, db, reqs, preset)
        for r, a in zip(reqs, alone):
            assert keys(r) == a
    finally:
        db.close()


def test_server_stream_continuous_batching(tmp_path):
    w = synth.workload(2, n_queries=10, n_db=1200, seed_offset=33)
    dl, do = drgpu.concat(w.db)
    rng = np.random.Generator(np.random.PCG64(5))
    # the requests arrive together, so that queued requests of one preset are
    # admitted as one batch whatever the speed of the GPU
    stream = serve.poisson_stream(rng, 24, rate=1e6, max_queries=12,
                                  presets=["fast", "default", "sensitive", "very-sensitive"], q_hi=600)
    srv = serve.Server(dl, do, workers=2, batch=True, index_budget=1 << 30, tune_cache=str(tmp_path / "tune.txt"))
    try:
        # grows scratch, builds two presets' indexes and autotunes them (the
        # other presets run with the base tuning)
        srv.warm(["fast", "very-sensitive"], w.queries[:3])
        assert set(srv.tunings) == {"fast", "very-sensitive"}
        assert (tmp_path / "tune.txt").read_text().count("\n") == 2
        finished, span = serve.run_stream(srv, stream)
    finally:
        srv.close()
    assert len(finished) == len(stream)
    assert max(r.batch_size for r in finished) >= 2  # requests were admitted together
    summary = serve.latency_summary(finished, span)
    assert summary["p50_s"] <= summary["p99_s"]
    ctx = drgpu.Context(0)
    db = drgpu.ResidentDb(ctx, dl, do)
    try:
        for r in finished:
            assert keys(r) == solo(ctx, db, r, r.preset), (r.rid, r.preset, r.batch_size)
    finally:
        db.close()
        ctx.close()
