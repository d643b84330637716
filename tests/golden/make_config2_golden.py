#!/usr/bin/env python3
"""Golden HSP lists of the timed benchmark batch, made by the CPU oracle.

The benchmark times one search of 1,000 synthetic queries (lognormal mean 350,
50-1500 aa, 5 planted homologs each) against a 7,860-sequence synthetic
database, blastp --sensitive and --very-sensitive, index-chunks 1.  The seed
join's expansion cap counts query occurrences over the whole batch
(seed.rs:120-127, search.rs:109-131), so the batch has to be compared as one
search; the oracle needs minutes for it, so its answer is kept here.

Writes config2_<preset>.jsonl.gz: one JSON array per HSP in the order of the
per-target lists (target, then the fields of drgpu.HspRecord.key(), floats as
exact reprs), plus config2_<preset>.sha256 of the uncompressed text.

Usage: python tests/golden/make_config2_golden.py [--threads N] [preset ...]
"""
import argparse
import gzip
import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "diamond-rust_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def canonical_lines(lists):
    """One line per HSP: [target, query, subject, frame, score, q_begin, q_end,
    s_begin, s_end, bits, evalue, identities, positives, mismatches,
    gap_openings, gaps, length, [ops...]] (floats by repr: exact)."""
    out = []
    for t, lst in enumerate(lists):
        for h in lst:
            row = [t] + [x for x in h[:16]] + [list(h[16])]
            out.append(json.dumps(row, separators=(",", ":")))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("presets", nargs="*", default=["sensitive", "very-sensitive"])
    a = ap.parse_args()
    import pyoracle
    from drgpu import synth
    w = synth.workload(2)
    for preset in a.presets:
        t0 = time.time()
        lists, stats = pyoracle.search(w.db, w.queries, sensitivity=preset, index_chunks=1, threads=a.threads)
        lines = canonical_lines(lists)
        text = "\n".join(lines) + "\n"
        name = f"config2_{preset}"
        with gzip.GzipFile(os.path.join(HERE, name + ".jsonl.gz"), "wb", mtime=0) as f:
            f.write(text.encode())
        digest = hashlib.sha256(text.encode()).hexdigest()
        with open(os.path.join(HERE, name + ".sha256"), "w") as f:
            f.write(f"{digest}  {len(lines)} hsps  hits {stats['hits']}\n")
        print(f"{preset}: {len(lines)} HSPs, {stats['hits']} hits, {time.time() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    main()
