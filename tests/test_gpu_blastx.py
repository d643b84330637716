"""blastx front end on the GPU (translate.rs:54-137, workflow.rs:112-127).

Six-frame translation, short-ORF masking and the drop of all-X frames run on
the device (drg_translate_reads / drg_batch_create_blastx); the frames must
equal the oracle's translate.rs restatement byte for byte, and a blastx search
over the device batch, merged per read (search::merge_frames), must equal the
oracle's search of the same frames.
"""
import numpy as np
import pytest

import drgpu
from drgpu import synth

pytestmark = pytest.mark.gpu


def oracle_frames(orc, reads, min_orf):
    """workflow.rs:112-127 over the oracle's translate.rs."""
    frames, query, frame = [], [], []
    for qi, r in enumerate(reads):
        m = orc.min_orf_len(len(r), None if min_orf < 0 else min_orf)
        for f, fr in enumerate(orc.six_frames(r)):
            fr = orc.mask_short_orfs(fr, m)
            if not (fr < 23).any():
                continue
            frames.append(fr)
            query.append(qi)
            frame.append(f)
    return frames, query, frame


def random_reads(r, n):
    alphabet = np.array(list("ACGT" * 12 + "NRYSWKMBVDHU" + "acgtn"))
    reads = []
    for k in range(n):
        L = int(r.choice([0, 1, 2, 3, 5, 29, 30, 31, 99, 100, 101])) if k % 4 == 0 else int(r.integers(0, 400))
        reads.append("".join(r.choice(alphabet, size=L)))
    return reads


@pytest.mark.parametrize("min_orf", [-1, 0, 1, 5, 60])
def test_translation_matches_oracle(ctx, orc, min_orf):
    r = np.random.Generator(np.random.PCG64(100 + min_orf))
    reads = random_reads(r, 300)
    # long stop-free and stop-rich reads
    reads.append("ATG" + "GCT" * 200)
    reads.append("TAA" * 50 + "GGG" * 30)
    got, q, f = ctx.translate_reads(reads, min_orf)
    exp, eq, ef = oracle_frames(orc, reads, min_orf)
    assert list(q) == eq and list(f) == ef
    assert len(got) == len(exp)
    for a, b in zip(got, exp):
        assert np.array_equal(a, b)


def test_translation_edge_cases(ctx, orc):
    got, q, f = ctx.translate_reads([], -1)
    assert got == [] and len(q) == 0
    got, q, f = ctx.translate_reads(["", "A", "AC"], -1)  # no codon in any frame
    assert got == []
    got, q, f = ctx.translate_reads(["NNNNNNNNN"], -1)  # every codon ambiguous: all frames dropped
    assert got == []
    # stops forward, leucines on the reverse strand; a two-codon read
    for reads in (["TAATAATAA"], ["ATGGCC"], ["TAATAATAA", "NNNNNNNNN", "ATGGCC"]):
        got, q, f = ctx.translate_reads(reads, -1)
        exp, eq, ef = oracle_frames(orc, reads, -1)
        assert [list(x) for x in got] == [list(x) for x in exp] and list(q) == eq and list(f) == ef


@pytest.mark.parametrize("preset", ["fast", "default"])
def test_blastx_search_on_device_frames(ctx, orc, preset):
    w = synth.read_workload(n_reads=200, n_db=1200, seed_offset=7)
    reads = w.reads
    dl, do = drgpu.concat(w.db)
    db = drgpu.ResidentDb(ctx, dl, do)
    batch = drgpu.blastx_batch(ctx, reads)
    try:
        cfg = drgpu.make_config(sensitivity=preset)
        lists, _, _ = drgpu.search_resident(ctx, db, batch, cfg, merge_queries=len(reads))
    finally:
        batch.close()
        db.close()
    frames, query, frame = oracle_frames(orc, reads, -1)
    assert list(batch.query) == query and list(batch.frame) == frame
    exp, _ = orc.search(w.db, frames, sensitivity=preset, t_query=np.array(query), t_frame=np.array(frame),
                        merge=True, n_queries=len(reads), threads=8)
    got = [[h.key() for h in lst] for lst in lists]
    assert got == exp
    assert sum(len(x) for x in exp) > 0
