"""Parity of the exact batch the benchmark times: 1,000 synthetic queries
against the 7,860-sequence synthetic database, blastp --sensitive and
--very-sensitive, index-chunks 1, searched as ONE batch through the resident
entry point the benchmark times (drg_search_batch).

The seed join's expansion cap counts each query seed key over the whole batch
(seed.rs:120-127, search.rs:109-131), so a sample searched on its own is a
different search; this compares every HSP of the whole batch, every field
bit for bit, with the oracle's answer for that batch
(tests/golden/config2_<preset>.jsonl.gz, made by make_config2_golden.py).
"""
import gzip
import hashlib
import json
import os

import pytest

import drgpu  # noqa: E402
from drgpu import synth  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PRESETS = ["sensitive", "very-sensitive"]


def golden_text(preset):
    with gzip.open(os.path.join(GOLDEN, f"config2_{preset}.jsonl.gz"), "rb") as f:
        return f.read().decode()


def golden_lists(preset, n_targets):
    lists = [[] for _ in range(n_targets)]
    for line in golden_text(preset).splitlines():
        row = json.loads(line)
        lists[row[0]].append(tuple(row[1:17]) + (tuple(row[17]),))
    return lists


@pytest.mark.parametrize("preset", PRESETS)
def test_golden_fixture_intact(preset):
    with open(os.path.join(GOLDEN, f"config2_{preset}.sha256")) as f:
        digest, n = f.read().split()[:2]
    text = golden_text(preset)
    assert hashlib.sha256(text.encode()).hexdigest() == digest
    assert len(text.splitlines()) == int(n)


@pytest.fixture(scope="module")
def resident(ctx):
    w = synth.workload(2)
    dl, do = drgpu.concat(w.db)
    tl, to = drgpu.concat(w.queries)
    db = drgpu.ResidentDb(ctx, dl, do)
    batch = drgpu.ResidentBatch(ctx, tl, to)
    yield w, db, batch
    batch.close()
    db.close()


@pytest.mark.gpu
@pytest.mark.parametrize("preset", PRESETS)
def test_timed_batch_matches_oracle(ctx, resident, preset):
    w, db, batch = resident
    cfg = drgpu.make_config(sensitivity=preset, index_chunks=1)
    got, stats = drgpu.search_resident(ctx, db, batch, cfg)[:2]
    exp = golden_lists(preset, len(w.queries))
    got_t = [[h.key() for h in lst] for lst in got]
    assert len(got_t) == len(exp)
    bad = [t for t in range(len(exp)) if got_t[t] != exp[t]]
    assert not bad, f"{len(bad)} targets differ, first {bad[:5]}"
    assert sum(len(x) for x in exp) > 4000
