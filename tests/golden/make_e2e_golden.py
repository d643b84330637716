#!/usr/bin/env python3
"""Outfmt 6 lines of the CPU oracle on the reference's own end-to-end data.

The reference ships bench/e2e/db_prot.fa (7,860 proteins, 2,263,996 aa) and
bench/e2e/query.fa (one 497-aa query) and publishes, in its README, the hit
counts and a few fields of blastp on them.  This script runs the oracle's
command line (makedb, then blastp for five presets) on that data and keeps the
tabular lines in e2e_outfmt6.txt, one block per preset, so that the published
answers are checked (tests/test_oracle_known_answers.py) where the data set is
not mounted.

Usage: python tests/golden/make_e2e_golden.py E2E_DIR
       (E2E_DIR = the reference's bench/e2e directory; build the oracle first)
"""
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
ORACLE = os.path.join(ROOT, "oracle", "_build", "oracle")
PRESETS = ["default", "fast", "sensitive", "more-sensitive", "very-sensitive"]


def run(e2e):
    out = []
    with tempfile.TemporaryDirectory() as d:
        db = os.path.join(d, "db_prot")
        subprocess.run([ORACLE, "makedb", "--in", os.path.join(e2e, "db_prot.fa"), "-d", db, "--quiet"],
                       check=True, capture_output=True, timeout=300)
        for preset in PRESETS:
            args = [ORACLE, "blastp", "-d", db, "-q", os.path.join(e2e, "query.fa"), "--quiet"]
            if preset != "default":
                args.append(f"--{preset}")
            r = subprocess.run(args, check=True, capture_output=True, text=True, timeout=600)
            out.append(f"# {preset}")
            out.extend(r.stdout.splitlines())
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    lines = run(sys.argv[1])
    with open(os.path.join(HERE, "e2e_outfmt6.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    print(f"{len(lines)} lines")


if __name__ == "__main__":
    main()
