"""The drop-in boundary on a host without a GPU (CPU only).

The C-ABI library loads, exports every function include/drgpu.h declares,
answers its host-only calls like the oracle, and refuses to create a device
context when no CUDA device is present (there is no CPU fallback).
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

import drgpu
import pyoracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "drgpu.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(drg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = C.CDLL(drgpu.LIB_PATH)
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []
    # the Python binding declares a signature for each of them
    assert sorted(drgpu.exported_symbols()) == names


def test_index_budget_on_a_null_db_is_an_error():
    lib = drgpu.load_library()
    assert lib.drg_db_set_index_budget(None, 1) == 1  # DRG_ERR_INVALID
    assert lib.drg_db_index_stats(None, None) == 1


def test_version_names_the_target():
    lib = drgpu.load_library()
    assert b"sm_100a" in lib.drg_version()


def test_no_device_is_a_loud_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = drgpu.load_library()
    h = C.c_void_p()
    rc = lib.drg_ctx_create(0, C.byref(h))
    assert rc == 6  # DRG_ERR_NODEVICE
    with pytest.raises(drgpu.DrgError):
        drgpu.Context(0)


@pytest.mark.parametrize("n,parts", [(0, 4), (1, 4), (10, 4), (7, 3), (7860, 4), (100, 1), (5, 9)])
def test_seed_chunks_match_oracle(n, parts):
    lib = drgpu.load_library()
    out = (C.c_uint64 * (2 * parts + 2))()
    k = C.c_uint64()
    assert lib.drg_seed_chunks(n, parts, out, C.byref(k)) == 0
    got = [(out[2 * i], out[2 * i + 1]) for i in range(k.value)]
    assert got == orc.chunks(n, parts)


@pytest.mark.parametrize("matrix,go,ge", [("BLOSUM62", -1, -1), ("BLOSUM62", 9, 2), ("BLOSUM45", -1, -1),
                                          ("BLOSUM50", -1, -1), ("BLOSUM80", -1, -1), ("BLOSUM90", -1, -1),
                                          ("PAM250", -1, -1), ("PAM70", -1, -1), ("PAM30", -1, -1)])
def test_matrix_evalue_bit_exact_with_oracle(matrix, go, ge):
    rng = np.random.default_rng(7)
    for _ in range(300):
        raw = int(rng.integers(1, 3000))
        qlen = int(rng.integers(1, 5000))
        slen = int(rng.integers(1, 5000))
        db = int(rng.integers(1, 10**10))
        e, b = drgpu.matrix_evalue(raw, qlen, slen, db, matrix, go, ge)
        assert e == orc.evalue(raw, qlen, slen, db, matrix, go, ge)
        assert b == orc.bit_score(raw, matrix, go, ge)


def test_matrix_evalue_rejects_unknown_inputs():
    with pytest.raises(drgpu.DrgError):
        drgpu.matrix_evalue(100, 300, 300, 10**6, "NOPE")
    with pytest.raises(drgpu.DrgError):
        drgpu.matrix_evalue(100, 300, 300, 10**6, "BLOSUM62", 42, 7)
