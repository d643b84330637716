"""The drop-in command line (bin/drgpu) against the oracle's command line.

CPU: makedb writes byte-identical DRDMND01 files, dbinfo prints the same
report, option errors and the missing-GPU error are loud.  GPU: blastp and
blastx print byte-identical --outfmt 6 output (default columns and every
field the reference knows) for the sensitivity presets.
"""
import os
import subprocess

import pytest

from drgpu import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "diamond-rust_b200", "bin", "drgpu")
ORACLE = os.path.join(ROOT, "oracle", "_build", "oracle")

ALL_FIELDS = ("qseqid qlen sseqid slen qstart qend sstart send qseq sseq evalue bitscore score length pident nident "
              "mismatch positive gapopen gaps ppos qframe qcovhsp scovhsp cigar btop qtitle stitle full_sseq "
              "qseq_translated qstrand").split()


def run(exe, *args, cwd=None):
    return subprocess.run([exe, *args], capture_output=True, text=True, cwd=cwd, timeout=900)


def has_gpu():
    import torch
    return torch.cuda.is_available()


@pytest.fixture(scope="module")
def config1_files(tmp_path_factory):
    d = tmp_path_factory.mktemp("cfg1")
    w = synth.workload(1)
    db_fa, q_fa = str(d / "db.fa"), str(d / "q.fa")
    w.write_fasta(db_fa, q_fa)
    return d, db_fa, q_fa


def test_makedb_is_byte_identical(config1_files):
    d, db_fa, _ = config1_files
    a = run(CLI, "makedb", "--in", db_fa, "-d", str(d / "mine"))
    b = run(ORACLE, "makedb", "--in", db_fa, "-d", str(d / "theirs"))
    assert a.returncode == 0 and b.returncode == 0, a.stderr + b.stderr
    assert open(d / "mine.dmnd", "rb").read() == open(d / "theirs.dmnd", "rb").read()
    assert "Sequences: 7860" in a.stderr


def test_dbinfo_matches(config1_files):
    d, db_fa, _ = config1_files
    run(CLI, "makedb", "--in", db_fa, "-d", str(d / "info"), "--quiet")
    a = run(CLI, "dbinfo", "--db", str(d / "info"))
    b = run(ORACLE, "dbinfo", "--db", str(d / "info"))
    assert a.returncode == 0 and a.stdout == b.stdout


def test_makedb_edge_inputs(tmp_path):
    fa = tmp_path / "x.fa"
    fa.write_text(">a desc\r\nac-de.f\n\n; comment\n>b\n\n>c  \nWWW*X\n")
    for exe, name in ((CLI, "m"), (ORACLE, "o")):
        r = run(exe, "makedb", "--in", str(fa), "--db", str(tmp_path / name), "--no-auto-append", "--quiet")
        assert r.returncode == 0, r.stderr
    assert (tmp_path / "m").read_bytes() == (tmp_path / "o").read_bytes()
    bad = tmp_path / "bad.fa"
    bad.write_text("ACGT\n>a\nAC\n")
    r = run(CLI, "makedb", "--in", str(bad), "--db", str(tmp_path / "bad"))
    assert r.returncode == 1 and "before the first '>' header" in r.stderr


@pytest.mark.parametrize("args,msg", [
    (["blastp", "-q", "q.fa"], "Missing option: --db"),
    (["blastp", "-d", "nr"], "Missing option: --query"),
    (["makedb", "-i", "x.fa"], "Missing option: --db"),
    (["blastp", "-d", "nr", "-q", "q.fa", "--nope"], "Unknown option: --nope"),
    (["blastp", "-d", "nr", "-q", "q.fa", "-k", "ten"], "Invalid value for --k"),
    (["frobnicate"], "Unknown command: frobnicate"),
])
def test_option_errors(args, msg):
    r = run(CLI, *args)
    assert r.returncode == 1
    assert msg in r.stderr


def test_version_and_usage():
    r = run(CLI, "version")
    assert r.returncode == 0 and "diamond-rust" in r.stdout
    r = run(CLI, "help")
    for cmd in ("makedb", "blastp", "blastx", "dbinfo"):
        assert cmd in r.stdout


def test_no_gpu_is_a_loud_error(config1_files):
    if has_gpu():
        pytest.skip("a CUDA device is present")
    d, db_fa, q_fa = config1_files
    run(CLI, "makedb", "--in", db_fa, "-d", str(d / "nogpu"), "--quiet")
    r = run(CLI, "blastp", "-d", str(d / "nogpu"), "-q", q_fa)
    assert r.returncode == 1 and "no CUDA device" in r.stderr and r.stdout == ""


# ---- GPU: outfmt 6 byte parity ---------------------------------------------------------------


def _blast_pair(kind, db, q, extra):
    a = run(CLI, kind, "-d", db, "-q", q, "--quiet", *extra)
    b = run(ORACLE, kind, "-d", db, "-q", q, "--quiet", *extra)
    assert a.returncode == 0, a.stderr
    assert b.returncode == 0, b.stderr
    return a.stdout, b.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("preset", ["fast", "default", "sensitive", "more-sensitive", "very-sensitive"])
def test_blastp_config1_outfmt6_identical(config1_files, preset):
    d, db_fa, q_fa = config1_files
    db = str(d / "p1")
    run(CLI, "makedb", "--in", db_fa, "-d", db, "--quiet")
    flag = [] if preset == "default" else [f"--{preset}"]
    mine, theirs = _blast_pair("blastp", db, q_fa, flag)
    assert mine == theirs
    assert len(mine.splitlines()) >= 1
    mine, theirs = _blast_pair("blastp", db, q_fa, flag + ["--outfmt", "6", *ALL_FIELDS])
    assert mine == theirs


@pytest.mark.gpu
def test_blastp_many_queries_options_identical(tmp_path):
    w = synth.workload(2, n_queries=40, n_db=1500, seed_offset=11)
    db_fa, q_fa = str(tmp_path / "db.fa"), str(tmp_path / "q.fa")
    w.write_fasta(db_fa, q_fa)
    db = str(tmp_path / "db")
    run(CLI, "makedb", "--in", db_fa, "-d", db, "--quiet")
    for extra in (["--sensitive", "-k", "5", "--max-hsps", "3", "-e", "1e-5"],
                  ["--matrix", "BLOSUM45", "--index-chunks", "2"],
                  ["--very-sensitive", "--outfmt", "6", "qseqid", "sseqid", "btop", "cigar", "qseq", "sseq"]):
        mine, theirs = _blast_pair("blastp", db, q_fa, extra)
        assert mine == theirs, extra
    out = tmp_path / "hits.tsv"
    r = run(CLI, "blastp", "-d", db, "-q", q_fa, "--quiet", "-o", str(out))
    assert r.returncode == 0 and r.stdout == ""
    assert out.read_text() == _blast_pair("blastp", db, q_fa, [])[1]


@pytest.mark.gpu
@pytest.mark.parametrize("preset", ["fast", "default"])
def test_blastx_reads_outfmt6_identical(tmp_path, preset):
    w = synth.read_workload(n_reads=300, n_db=800, seed_offset=3)
    db_fa, r_fa = str(tmp_path / "db.fa"), str(tmp_path / "reads.fa")
    w.write_fasta(db_fa, r_fa)
    db = str(tmp_path / "db")
    run(CLI, "makedb", "--in", db_fa, "-d", db, "--quiet")
    flag = [] if preset == "default" else [f"--{preset}"]
    mine, theirs = _blast_pair("blastx", db, r_fa, flag + ["--outfmt", "6", *ALL_FIELDS])
    assert mine == theirs
    assert len(mine.splitlines()) > 10
