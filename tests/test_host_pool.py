"""The host thread pool behind the search's CPU-side steps (CPU only).

Compiles tests/pool_check.cpp against the library's header and runs it: every
index of every parallel_for is visited exactly once, across pool sizes, grains,
part limits and repeated calls.
"""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_pool_visits_every_index_once(tmp_path):
    exe = str(tmp_path / "pool_check")
    src = os.path.join(ROOT, "tests", "pool_check.cpp")
    inc = os.path.join(ROOT, "diamond-rust_b200", "csrc")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-I", inc, src, "-o", exe], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
