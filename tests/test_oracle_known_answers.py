"""The oracle against the reference's published end-to-end answers (CPU only).

The reference's README reports, for its bench/e2e data (7,860 proteins,
2,263,996 aa, one 497-aa query): 4 / 1 / 7 / 7 / 7 hits for --default /
--fast / --sensitive / --more-sensitive / --very-sensitive; under
--sensitive WP_048121137.1 aligns over 612 columns at 91.7 bits; under
--default WP_048121132.1 is reported at 26.2 % identity and 83.2 bits.
These tests run where that data set is mounted and skip elsewhere.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle", "_build", "oracle")
E2E = os.environ.get("DRG_REFERENCE_E2E", "/root/reference/bench/e2e")

pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(E2E, "db_prot.fa")),
                                reason="the reference's bench/e2e data is not mounted here")


@pytest.fixture(scope="module")
def e2e_db(tmp_path_factory):
    d = tmp_path_factory.mktemp("e2e")
    db = str(d / "db_prot")
    r = subprocess.run([ORACLE, "makedb", "--in", os.path.join(E2E, "db_prot.fa"), "-d", db, "--quiet"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return db


def blastp(db, preset):
    args = [ORACLE, "blastp", "-d", db, "-q", os.path.join(E2E, "query.fa"), "--quiet"]
    if preset != "default":
        args.append(f"--{preset}")
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return [line.split("\t") for line in r.stdout.splitlines()]


@pytest.mark.parametrize("preset,hits", [("default", 4), ("fast", 1), ("sensitive", 7), ("more-sensitive", 7),
                                         ("very-sensitive", 7)])
def test_hit_counts(e2e_db, preset, hits):
    assert len(blastp(e2e_db, preset)) == hits


def test_sensitive_612_columns(e2e_db):
    rows = {r[1]: r for r in blastp(e2e_db, "sensitive")}
    r = rows["WP_048121137.1"]
    assert r[3] == "612"
    assert r[11] == "91.7"


def test_default_extra_hit(e2e_db):
    rows = {r[1]: r for r in blastp(e2e_db, "default")}
    r = rows["WP_048121132.1"]
    assert r[2] == "26.2"
    assert r[11] == "83.2"
