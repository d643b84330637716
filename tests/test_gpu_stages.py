"""Stage parity on the GPU: each C-ABI entry point against the CPU oracle.

seed::build, seed::join_into, ungapped::xdrop and gapped::extend_span are
compared on seeded random inputs and on the reference's own unit-test
vectors; everything is integer work, so the bar is exact equality.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import drgpu  # noqa: E402
from drgpu import synth  # noqa: E402


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def rand_seq(r, n, ambiguous=0.0):
    s = synth.random_protein(r, n)
    if ambiguous > 0 and n > 0:
        mask = r.random(n) < ambiguous
        s[mask] = r.integers(20, 25, size=int(mask.sum()))
    return s


# ---------------------------------------------------------------- seed::build
SHAPES = ["1111", "101", "111101110111", "1011110111", "11110111", "1101110101101111", "1100010100000010011",
          "1" + "0" * 40 + "111"]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("reduction", [0, 1, 2])
def test_seed_build_matches_oracle(ctx, orc, shape, reduction):
    r = rng(11 + len(shape) + reduction)
    seqs = [rand_seq(r, int(n), ambiguous=0.02) for n in r.integers(0, 120, size=40)]
    seqs[3] = np.full(60, 5, np.uint8)  # homopolymer: rejected by the complexity cut
    w = shape.count("1")
    for cut in (0.0, 0.8 * np.log(2) * w, 1.0 * np.log(2) * w):
        got = np.sort(ctx.seed_build(seqs, shape, reduction, base=7, cut=cut), order=["key", "seq", "pos"])
        exp = np.sort(orc.seed_build(seqs, shape, reduction, base=7, cut=cut), order=["key", "seq", "pos"])
        assert len(got) == len(exp)
        assert (got == exp).all()


def test_seed_build_reference_vectors(ctx, orc):
    # seed.rs:175-196: identical 10-mers give 7 seeds with the scaled default cut
    a = orc.encode("MKWVTFGCPD")
    cut = 0.8 * np.log(2) * 4
    assert len(ctx.seed_build([a], "1111", 0, 0, cut)) == 7
    # seed.rs:198-209 on 8-mers: homopolymer and AAAAAACC rejected by the scaled cut
    cut8 = 0.8 * np.log(2) * 8
    assert len(ctx.seed_build([orc.encode("AAAAAAAA")], "11111111", 0, 0, cut8)) == 0
    assert len(ctx.seed_build([orc.encode("AAAAAACC")], "11111111", 0, 0, cut8)) == 0
    assert len(ctx.seed_build([orc.encode("AAAAAACC")], "11111111", 0, 0, 0.8)) == 1
    # shape.rs:231-247: contiguous key 12*400 + 11*20 + 17 under no reduction
    e = ctx.seed_build([orc.encode("MKWV")], "111", 2, 0, 0.0)
    assert int(np.sort(e["key"])[0]) in (12 * 400 + 11 * 20 + 17, 11 * 400 + 17 * 20 + 19)
    keys = set(int(k) for k in e["key"])
    assert 12 * 400 + 11 * 20 + 17 in keys


def test_seed_build_rejects_bad_shape(ctx):
    with pytest.raises(drgpu.DrgError) as ei:
        ctx.seed_build([np.zeros(10, np.uint8)], "1021")
    assert ei.value.code == 1
    with pytest.raises(drgpu.DrgError) as ei:  # positions are bytes: 256 at most
        ctx.seed_build([np.zeros(300, np.uint8)], "1" + "0" * 255 + "1")
    assert ei.value.code == 1


def test_seed_build_longest_span(ctx, orc):
    r = rng(19)
    seqs = [rand_seq(r, int(n)) for n in (0, 255, 256, 257, 300, 600)]
    shape = "11" + "0" * 252 + "11"  # span 256
    got = np.sort(ctx.seed_build(seqs, shape, 0, base=3, cut=0.0), order=["key", "seq", "pos"])
    exp = np.sort(orc.seed_build(seqs, shape, 0, base=3, cut=0.0), order=["key", "seq", "pos"])
    assert len(exp) == 1 + 2 + 45 + 345 and (got == exp).all()


def test_seed_complexity_cut_at_the_boundary(ctx, orc):
    # The device sums the entropy per letter and recomputes it in the
    # reference's bucket order only near the cut: cuts a few ulps around the
    # entropy of each count pattern of a 4-letter seed must decide as the
    # oracle does.
    words = ["AACC", "ACAC", "AAAC", "AACD", "ACDE", "AAAA", "CACA", "DCBA"]
    seqs = [orc.encode(w * 6) for w in words]
    for e in (np.log(6.0), np.log(4.0), np.log(12.0), np.log(24.0), 0.0):
        for k in range(-4, 5):
            cut = float(e)
            for _ in range(abs(k)):
                cut = float(np.nextafter(cut, np.inf if k > 0 else -np.inf))
            got = np.sort(ctx.seed_build(seqs, "1111", 2, base=0, cut=cut), order=["key", "seq", "pos"])
            exp = np.sort(orc.seed_build(seqs, "1111", 2, base=0, cut=cut), order=["key", "seq", "pos"])
            assert len(got) == len(exp) and (got == exp).all(), (e, k)


# ------------------------------------------------------------- seed::join_into
def test_join_matches_oracle(ctx, orc):
    r = rng(5)
    qs = [rand_seq(r, int(n)) for n in r.integers(45, 200, size=30)]
    rs = [rand_seq(r, int(n)) for n in r.integers(45, 300, size=60)]
    # shared low-complexity blocks make heavy keys on both sides (expansion cap)
    block = np.array([7, 7, 9, 7, 9, 9, 7, 7, 9, 7], np.uint8)
    for s in qs[:6]:
        s[:40] = np.tile(block, 4)
    for s in rs[:30]:
        s[:40] = np.tile(block, 4)
    for shape in ("1111", "110101"):
        qe = orc.seed_build(qs, shape, 0, 0, 0.0)
        re = orc.seed_build(rs, shape, 0, 100, 0.0)
        for cap in (4096, 64, 1):
            got = ctx.seed_join(qe, re, len(qs), cap)
            exp = orc.seed_join(qe, re, len(qs), cap)
            assert got == exp, (shape, cap)


def test_join_reference_vector(ctx, orc):
    a = orc.encode("MKWVTFGCPD")
    cut = 0.8 * np.log(2) * 4
    q = orc.seed_build([a], "1111", 0, 0, cut)
    r = orc.seed_build([a], "1111", 0, 7, cut)
    hits = ctx.seed_join(q, r, 1, 4096)
    assert len(hits) == 7
    assert all(h[2] == 7 for h in hits)
    assert sorted(hits, key=lambda h: h[1])[0][1:4:2] == (0, 0)


def test_chunks_match_oracle(orc):
    import ctypes as C
    lib = drgpu.load_library()
    for n, parts in [(10, 4), (0, 4), (7860, 4), (3, 8), (1, 1), (100, 0)]:
        out = (C.c_uint64 * 64)()
        k = C.c_uint64()
        assert lib.drg_seed_chunks(n, parts, out, C.byref(k)) == 0
        got = [(out[2 * i], out[2 * i + 1]) for i in range(k.value)]
        assert got == orc.chunks(n, parts)


# ------------------------------------------------------------ ungapped::xdrop
def test_xdrop_matches_oracle(ctx, orc):
    r = rng(17)
    queries, subjects, jobs = [], [], []
    for i in range(300):
        q = rand_seq(r, int(r.integers(1, 400)), ambiguous=0.01)
        s = synth.mutate(r, q, float(r.uniform(0.2, 1.0))) if i % 2 else rand_seq(r, int(r.integers(1, 400)))
        if len(s) == 0:
            s = rand_seq(r, 5)
        queries.append(q)
        subjects.append(s)
        jobs.append((i, i, int(r.integers(0, len(q) + 1)), int(r.integers(0, len(s) + 1))))
    for xd in (20, 5, 40, 1):
        got = ctx.xdrop(queries, subjects, jobs, xdrop=xd)
        exp = [orc.xdrop(queries[j[0]], subjects[j[1]], j[2], j[3], xd) for j in jobs]
        assert got == exp


def test_xdrop_reference_vectors(ctx, orc):
    # ungapped.rs:99-129
    q = orc.encode("MKWVTFISLLFLFSSAYSR")
    (seg,) = ctx.xdrop([q], [q], [(0, 0, 0, 0)], xdrop=40)
    assert seg[0] == 0 and seg[2] == len(q)
    q = orc.encode("WWWWWWWWWWCCCCCCCCCC")
    s = orc.encode("WWWWWWWWWWDDDDDDDDDD")
    (seg,) = ctx.xdrop([q], [s], [(0, 0, 0, 0)], xdrop=5)
    assert seg[2] == 10 and seg[3] == 110
    a = orc.encode("AAAAAA")
    (seg,) = ctx.xdrop([a], [a], [(0, 0, 0, 0)], xdrop=30)
    assert seg[:3] == (0, 0, 6)


# -------------------------------------------------------- gapped::extend_span
def span_cases(seed, n_cases, max_len=500):
    r = rng(seed)
    queries, subjects, jobs = [], [], []
    for i in range(n_cases):
        n = int(r.integers(0, max_len))
        q = rand_seq(r, n, ambiguous=0.01)
        kind = i % 4
        if kind == 0:
            s = rand_seq(r, int(r.integers(0, max_len)))
        elif kind in (1, 2):
            s = synth.mutate(r, q, float(r.uniform(0.3, 0.95))) if n else rand_seq(r, 10)
        else:
            s = np.concatenate([rand_seq(r, int(r.integers(0, 100))), synth.mutate(r, q, 0.6),
                                rand_seq(r, int(r.integers(0, 100)))]).astype(np.uint8)
        m = len(s)
        center = int(r.integers(-m - 20, n + 20)) if i % 5 else 0
        half = int(r.choice([0, 3, 8, 12, 16, 30, 40, 64, 64, 64, 100, 150]))
        d0, d1 = center - half, center + half + int(r.integers(0, 40))
        if i % 7 == 0:
            d0, d1 = d1, d0  # swapped bounds
        queries.append(q)
        subjects.append(s)
        jobs.append((i, i, d0, d1))
    return queries, subjects, jobs


def oracle_spans(orc, queries, subjects, jobs):
    return [orc.extend_span(queries[j[0]], subjects[j[1]], j[2], j[3])[0] for j in jobs]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_extend_span_exact_matches_oracle(ctx, orc, seed):
    queries, subjects, jobs = span_cases(seed, 250)
    got = ctx.extend_span(queries, subjects, jobs)
    exp = oracle_spans(orc, queries, subjects, jobs)
    for j, g, e in zip(jobs, got, exp):
        assert g == e, j


@pytest.mark.parametrize("seed", [4, 5, 6, 7])
def test_extend_span_packed_scores_match_oracle(ctx, orc, seed):
    queries, subjects, jobs = span_cases(seed, 400, max_len=700)
    scores, stats = ctx.extend_span_scores(queries, subjects, jobs)
    exp = oracle_spans(orc, queries, subjects, jobs)
    for j, g, e in zip(jobs, scores, exp):
        assert int(g) == (e[0] if e else 0), j
    assert stats["sw_launches"] >= 1


def test_packed_scores_on_search_like_bands(ctx, orc):
    """Many bands of one query (the warp-shared profile path), widths 25..129."""
    r = rng(99)
    queries, subjects, jobs = [], [], []
    qs = [rand_seq(r, L) for L in (37, 64, 140, 230, 351, 497, 900)]
    for qi, q in enumerate(qs):
        band = orc.band_for(len(q))
        for k in range(70):
            s = synth.mutate(r, q, 0.5) if k % 3 == 0 else rand_seq(r, int(r.integers(30, 800)))
            d = int(r.integers(-len(s) + 1, len(q)))
            subjects.append(s)
            jobs.append((qi, len(subjects) - 1, d - band, d + band))
    queries = qs
    scores, _ = ctx.extend_span_scores(queries, subjects, jobs)
    exp = [orc.extend_span(queries[j[0]], subjects[j[1]], j[2], j[3])[0] for j in jobs]
    for j, g, e in zip(jobs, scores, exp):
        assert int(g) == (e[0] if e else 0), j


def test_packed_scores_transposed_short_subjects(ctx, orc):
    """Bands on short subjects from long queries run with the subject as rows
    (fewer strips); a subject needs a warp's worth of such bands.  Widths mix
    narrow and medium (137..272) bands in one warp."""
    r = rng(123)
    queries = [rand_seq(r, int(L)) for L in r.integers(400, 1200, size=9)]
    subjects, jobs = [], []
    for k in range(3):
        m = int(r.integers(40, 140))
        base = queries[k][:m].copy() if k == 0 else rand_seq(r, m)
        subjects.append(synth.mutate(r, base, 0.3) if k == 0 else base)
        for t in range(60):
            qi = t % len(queries)
            n = len(queries[qi])
            half = int(r.choice([12, 16, 30, 40, 64, 80, 100]))
            d = int(r.integers(-m + 1, n))
            jobs.append((qi, k, d - half, d + half))
    # one subject with too few bands to be worth transposing
    subjects.append(rand_seq(r, 50))
    jobs += [(q, 3, -20, 20) for q in range(5)]
    scores, st = ctx.extend_span_scores(queries, subjects, jobs)
    exp = oracle_spans(orc, queries, subjects, jobs)
    for j, g, e in zip(jobs, scores, exp):
        assert int(g) == (e[0] if e else 0), j
    assert st["sw_transposed_bands"] >= 64


@pytest.mark.parametrize("matrix", ["BLOSUM45", "BLOSUM50", "BLOSUM80", "BLOSUM90", "PAM30", "PAM70", "PAM250"])
def test_packed_scores_other_matrices(ctx, orc, matrix):
    """The clamped column past row m + d1 (gapped.rs:86-92) can hold up to the
    matrix's largest score; packed bests up to that are recomputed exactly."""
    r = rng(7 + len(matrix))
    queries, subjects, jobs = span_cases(31 + len(matrix), 150, max_len=500)
    # C/C then W/W in the clamped column: in-band best 9..13, clamped cells up to 15/17
    queries.append(orc.encode("C" + "A" * 24 + "W" * 10 + "A" * 100))
    subjects.append(orc.encode("C" * 19 + "W"))
    jobs.append((len(queries) - 1, len(subjects) - 1, -5, 5))
    scores, _ = ctx.extend_span_scores(queries, subjects, jobs, matrix=matrix)
    exp = [orc.extend_span(queries[j[0]], subjects[j[1]], j[2], j[3], matrix=matrix)[0] for j in jobs]
    for j, g, e in zip(jobs, scores, exp):
        assert int(g) == (e[0] if e else 0), (matrix, j)
    got = ctx.extend_span(queries[-1:], subjects[-1:], [(0, 0, -5, 5)], matrix=matrix)
    assert got == [exp[-1]]


def test_letter_codes_above_24(ctx, orc):
    """Codes above 24 score as 24 (matrix.rs:164-168 clamps both indices) but
    count as identities only when equal (hsp.rs:46-56); the packed kernels
    read a clamped copy of the letters, the walk the letters as given."""
    r = rng(404)
    queries, subjects, jobs = [], [], []
    for k in range(60):
        q = rand_seq(r, int(r.integers(40, 400)))
        s = synth.mutate(r, q, 0.7) if k % 2 else rand_seq(r, int(r.integers(40, 400)))
        for seq in (q, s):
            mask = r.random(len(seq)) < 0.05
            seq[mask] = r.choice(np.array([24, 25, 26, 30, 99, 200, 255], np.uint8), size=int(mask.sum()))
        queries.append(q)
        subjects.append(s)
        half = int(r.choice([12, 30, 64, 100, 200]))
        d = int(r.integers(-20, 20))
        jobs.append((k, k, d - half, d + half))
    got = ctx.extend_span(queries, subjects, jobs)
    exp = oracle_spans(orc, queries, subjects, jobs)
    assert got == exp
    scores, _ = ctx.extend_span_scores(queries, subjects, jobs)
    assert [int(x) for x in scores] == [e[0] if e else 0 for e in exp]


def test_extend_span_edge_cases(ctx, orc):
    W = np.full(3100, 17, np.uint8)  # W/W scores 11: best 34100 does not fit 16 bits
    cases = [
        (orc.encode("MKWVTFISLLFLFSSAYSR"), orc.encode("MKWVTFISLLFLFSSAYSR"), -30, 30),
        (orc.encode("MKWVTFISLLFLFSSAYSR"), orc.encode("MKWVTFISLLLFSSAYSR"), -30, 30),
        (orc.encode("WWWWWWWWWW"), orc.encode("AAAAAAAAAA"), -15, 15),
        (np.zeros(0, np.uint8), orc.encode("AAAA"), -5, 5),
        (orc.encode("AAAA"), np.zeros(0, np.uint8), -5, 5),
        (orc.encode("ACDEFGHIKL"), orc.encode("ACDEFGHIKL"), 50, 80),     # band below the matrix
        (orc.encode("ACDEFGHIKL"), orc.encode("ACDEFGHIKL"), -80, -50),   # band right of the matrix
        (orc.encode("ACDEFGHIKLMNPQRSTVWY" * 5), orc.encode("ACDEFGHIKL"), 85, 95),  # virtual rows only
        (orc.encode("XXXXBJZ**ACD"), orc.encode("XXBZ*ACD"), -10, 10),
        # rows past m + d1 keep one clamped cell at column m; here they hold the best (W/W = 11)
        (orc.encode("A" * 25 + "W" * 10 + "A" * 100), orc.encode("C" * 19 + "W"), -5, 5),
        (orc.encode("A" * 25 + "W" * 10 + "A" * 100), orc.encode("C" * 19 + "W"), -30, 30),
        (W, W, -64, 64),
        (W[:2000], W[:2000], -20, 20),
    ]
    queries = [c[0] for c in cases]
    subjects = [c[1] for c in cases]
    jobs = [(i, i, c[2], c[3]) for i, c in enumerate(cases)]
    got = ctx.extend_span(queries, subjects, jobs)
    exp = oracle_spans(orc, queries, subjects, jobs)
    assert got == exp
    scores, _ = ctx.extend_span_scores(queries, subjects, jobs)
    assert [int(x) for x in scores] == [e[0] if e else 0 for e in exp]
    # gapped.rs:299-322: identical sequences align end to end; a deletion opens a gap
    assert got[0][1:5] == (0, 19, 0, 19) and got[0][7] == 0 and got[0][9] == 0
    assert got[1][9] > 0 and got[2] is None
    assert got[9][0] == 11  # the clamped column, not an in-band cell
    assert got[11][0] == 3100 * 11


def test_stage_errors(ctx):
    with pytest.raises(drgpu.DrgError):
        ctx.extend_span([np.zeros(5, np.uint8)], [np.zeros(5, np.uint8)], [(0, 3, 0, 1)])
    with pytest.raises(drgpu.DrgError):
        ctx.extend_span([np.zeros(5, np.uint8)], [np.zeros(5, np.uint8)], [(0, 0, 0, 1)], matrix="NOPE")
    with pytest.raises(drgpu.DrgError):
        ctx.xdrop([np.zeros(5, np.uint8)], [np.zeros(5, np.uint8)], [(0, 0, 9, 0)])
