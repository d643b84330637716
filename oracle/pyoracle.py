"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is a plain C++ restatement of the diamond-rust search path; this
module exposes it to the tests, the smoke check and the bench's CPU baseline.
Nothing in the product imports it.  Return shapes match drgpu's binding so
results can be compared directly.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
CLI = os.path.join(HERE, "_build", "oracle")


def build():
    subprocess.run(["make", "-s", "-C", HERE, "-j8"], check=True)


class _Seg(C.Structure):
    _fields_ = [("q_start", C.c_uint64), ("s_start", C.c_uint64), ("len", C.c_uint64), ("score", C.c_int32),
                ("pad", C.c_int32)]


class _Aligned(C.Structure):
    _fields_ = [("found", C.c_int32), ("score", C.c_int32), ("q_begin", C.c_uint64), ("q_end", C.c_uint64),
                ("s_begin", C.c_uint64), ("s_end", C.c_uint64), ("identities", C.c_uint32),
                ("positives", C.c_uint32), ("mismatches", C.c_uint32), ("gap_openings", C.c_uint32),
                ("gaps", C.c_uint32), ("length", C.c_uint32), ("cells", C.c_uint64), ("n_ops", C.c_uint32),
                ("pad", C.c_uint32)]


class _Entry(C.Structure):
    _fields_ = [("key", C.c_uint64), ("seq", C.c_uint32), ("pos", C.c_uint32)]


class _Hit(C.Structure):
    _fields_ = [("query", C.c_uint32), ("qpos", C.c_uint32), ("subject", C.c_uint32), ("spos", C.c_uint32)]


class _Hsp(C.Structure):
    _fields_ = [("query", C.c_uint32), ("subject", C.c_uint32), ("frame", C.c_uint32), ("score", C.c_int32),
                ("q_begin", C.c_uint32), ("q_end", C.c_uint32), ("s_begin", C.c_uint32), ("s_end", C.c_uint32),
                ("bits", C.c_double), ("evalue", C.c_double), ("identities", C.c_uint32),
                ("positives", C.c_uint32), ("mismatches", C.c_uint32), ("gap_openings", C.c_uint32),
                ("gaps", C.c_uint32), ("length", C.c_uint32), ("ops_offset", C.c_uint64), ("n_ops", C.c_uint32),
                ("pad", C.c_uint32)]


class _Cfg(C.Structure):
    _fields_ = [("matrix", C.c_char_p), ("gap_open", C.c_int32), ("gap_extend", C.c_int32), ("evalue", C.c_double),
                ("max_target_seqs", C.c_uint32), ("max_hsps", C.c_uint32), ("sensitivity", C.c_char_p),
                ("index_chunks", C.c_int32), ("has_seed_cut", C.c_int32), ("seed_cut", C.c_double),
                ("threads", C.c_uint32), ("pad", C.c_uint32)]


class _Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("query_seeds", "ref_seeds", "hits", "xdrops", "segments", "bands",
                                          "dp_cells", "hsps")] + [("t_seed_join", C.c_double),
                                                                  ("t_align", C.c_double),
                                                                  ("clipped_windows", C.c_uint64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        _lib.orc_evalue.restype = C.c_double
        _lib.orc_evalue.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_size_t, C.c_size_t, C.c_uint64]
        _lib.orc_bit_score.restype = C.c_double
        _lib.orc_bit_score.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int]
        _lib.orc_raw_score.restype = C.c_int
        _lib.orc_raw_score.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_double]
        _lib.orc_log_erfc.restype = C.c_double
        _lib.orc_log_erfc.argtypes = [C.c_double]
        _lib.orc_ln_factorial.restype = C.c_double
        _lib.orc_ln_factorial.argtypes = [C.c_int]
        _lib.orc_band_for.restype = C.c_size_t
        _lib.orc_band_for.argtypes = [C.c_size_t]
        _lib.orc_last_error.restype = C.c_char_p
        _lib.orc_fmt_evalue.argtypes = [C.c_double, C.c_char_p, C.c_size_t]
        _lib.orc_fmt_double.argtypes = [C.c_double, C.c_char_p, C.c_size_t]
        _lib.orc_seed_is_complex.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_double]
        _lib.orc_shape_packed.argtypes = [C.c_char_p, C.c_size_t, C.c_size_t, C.c_char_p, C.c_int,
                                          C.POINTER(C.c_uint64)]
        _lib.orc_encode.restype = C.c_size_t
        _lib.orc_encode.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p]
        _lib.orc_free.argtypes = [C.c_void_p]
        _lib.orc_decode.restype = C.c_size_t
        _lib.orc_decode.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t]
        _lib.orc_seq_id.restype = C.c_size_t
        _lib.orc_seq_id.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t]
        _lib.orc_bucket.argtypes = [C.c_int, C.c_uint8, C.POINTER(C.c_uint64)]
        _lib.orc_reduction_size_for.restype = C.c_uint64
        _lib.orc_reduction_size_for.argtypes = [C.c_char_p]
        _lib.orc_seed_cut_for.restype = C.c_double
        _lib.orc_seed_cut_for.argtypes = [C.c_char_p, C.c_int, C.c_double]
        _lib.orc_index_chunks_for.restype = C.c_size_t
        _lib.orc_index_chunks_for.argtypes = [C.c_char_p, C.c_long]
        _lib.orc_translate_frame.restype = C.c_size_t
        _lib.orc_translate_frame.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t]
        _lib.orc_six_frames.restype = C.c_size_t
        _lib.orc_six_frames.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_uint64)]
        _lib.orc_mask_short_orfs.argtypes = [C.c_char_p, C.c_size_t, C.c_size_t]
        _lib.orc_min_orf_len.restype = C.c_size_t
        _lib.orc_min_orf_len.argtypes = [C.c_size_t, C.c_long]
        _lib.orc_parse_outfmt.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.c_int]
        _lib.orc_q_frame.argtypes = [C.c_uint32]
        _lib.orc_nt_range.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]
        _lib.orc_evalue_blast.restype = C.c_double
        _lib.orc_evalue_blast.argtypes = [C.c_char_p, C.c_int, C.c_size_t, C.c_uint64]
        _lib.orc_matrix_ok.argtypes = [C.c_char_p, C.c_int, C.c_int]
    return _lib


def decode(letters) -> str:
    b = C.create_string_buffer(len(letters) + 1)
    n = lib().orc_decode(_bytes(letters) if len(letters) else b"\0", len(letters), b, len(letters) + 1)
    return b.raw[:n].decode()


def seq_id(header: str) -> str:
    b = C.create_string_buffer(len(header) + 1)
    n = lib().orc_seq_id(header.encode(), b, len(header) + 1)
    return b.raw[:n].decode()


REDUCTIONS = {"murphy10": 0, "diamond9": 1, "none": 2}


def bucket(reduction: str, letter: int):
    size = C.c_uint64()
    b = lib().orc_bucket(REDUCTIONS[reduction], letter, C.byref(size))
    return b, size.value


def reduction_size_for(sens: str) -> int:
    return lib().orc_reduction_size_for(sens.encode())


def seed_cut_for(sens: str, cut=None) -> float:
    return lib().orc_seed_cut_for(sens.encode(), cut is not None, 0.0 if cut is None else cut)


def index_chunks_for(sens: str, chunks=None) -> int:
    return lib().orc_index_chunks_for(sens.encode(), -1 if chunks is None else chunks)


def translate_frame(nt: str, offset: int) -> np.ndarray:
    b = C.create_string_buffer(len(nt) // 3 + 1)
    n = lib().orc_translate_frame(nt.encode(), offset, b, len(nt) // 3 + 1)
    return np.frombuffer(b.raw[:n], dtype=np.uint8).copy()


def six_frames(nt: str):
    cap = 2 * len(nt) + 6
    b = C.create_string_buffer(cap)
    lens = (C.c_uint64 * 6)()
    lib().orc_six_frames(nt.encode(), b, cap, lens)
    out, k = [], 0
    for i in range(6):
        out.append(np.frombuffer(b.raw[k:k + lens[i]], dtype=np.uint8).copy())
        k += lens[i]
    return out


def mask_short_orfs(frame, min_len) -> np.ndarray:
    b = C.create_string_buffer(_bytes(frame), len(frame))
    lib().orc_mask_short_orfs(b, len(frame), min_len)
    return np.frombuffer(b.raw[:len(frame)], dtype=np.uint8).copy()


def min_orf_len(dna_len, user=None) -> int:
    return lib().orc_min_orf_len(dna_len, -1 if user is None else user)


FIELD_NAMES = ["qseqid", "qlen", "sseqid", "slen", "qstart", "qend", "sstart", "send", "qseq", "sseq", "evalue",
               "bitscore", "score", "length", "pident", "nident", "mismatch", "positive", "gapopen", "gaps", "ppos",
               "qframe", "qcovhsp", "scovhsp", "cigar", "btop", "qtitle", "stitle", "full_sseq", "qseq_translated",
               "qstrand"]


def parse_outfmt(tokens):
    """Field names of an --outfmt token list, or None when the reference rejects it."""
    f = (C.c_int * 64)()
    n = lib().orc_parse_outfmt(" ".join(tokens).encode(), f, 64)
    return None if n < 0 else [FIELD_NAMES[f[i]] for i in range(n)]


def q_frame(frame: int) -> int:
    return lib().orc_q_frame(frame)


def nt_range(frame, q_begin, q_end, dna_len):
    o = (C.c_uint64 * 2)()
    lib().orc_nt_range(frame, q_begin, q_end, dna_len, o)
    return (o[0], o[1])


def evalue_blast(raw, qlen, db, matrix="BLOSUM62"):
    return lib().orc_evalue_blast(matrix.encode(), raw, qlen, db)


def matrix_ok(matrix, go=-1, ge=-1) -> bool:
    return bool(lib().orc_matrix_ok(matrix.encode(), go, ge))


def _bytes(a):
    return np.ascontiguousarray(a, dtype=np.uint8).tobytes()


def concat(seqs):
    off = np.zeros(len(seqs) + 1, dtype=np.uint64)
    if len(seqs):
        off[1:] = np.cumsum([len(s) for s in seqs])
    letters = np.concatenate([np.asarray(s, np.uint8) for s in seqs]) if len(seqs) else np.zeros(1, np.uint8)
    if len(letters) == 0:
        letters = np.zeros(1, np.uint8)
    return np.ascontiguousarray(letters, np.uint8), off


def encode(text: str) -> np.ndarray:
    out = C.create_string_buffer(len(text) + 1)
    n = lib().orc_encode(text.encode(), len(text), out)
    return np.frombuffer(out.raw[:n], dtype=np.uint8).copy()


def evalue(raw, qlen, slen, db, matrix="BLOSUM62", go=-1, ge=-1):
    return lib().orc_evalue(matrix.encode(), go, ge, raw, qlen, slen, db)


def bit_score(raw, matrix="BLOSUM62", go=-1, ge=-1):
    return lib().orc_bit_score(matrix.encode(), go, ge, raw)


def raw_score(bits, matrix="BLOSUM62", go=-1, ge=-1):
    return lib().orc_raw_score(matrix.encode(), go, ge, bits)


def log_erfc(x):
    return lib().orc_log_erfc(x)


def ln_factorial(n):
    return lib().orc_ln_factorial(n)


def band_for(n):
    return lib().orc_band_for(n)


def fmt_evalue(e):
    b = C.create_string_buffer(64)
    lib().orc_fmt_evalue(e, b, 64)
    return b.value.decode()


def fmt_double(x):
    b = C.create_string_buffer(64)
    lib().orc_fmt_double(x, b, 64)
    return b.value.decode()


def shapes_for(sens):
    b = C.create_string_buffer(4096)
    n = lib().orc_shapes_for(sens.encode(), b, 4096)
    return b.value.decode().split(",")[:n]


def chunks(n, parts):
    out = (C.c_uint64 * (2 * max(parts, 1) + 2))()
    k = lib().orc_chunks(C.c_size_t(n), C.c_size_t(parts), out)
    return [(out[2 * i], out[2 * i + 1]) for i in range(k)]


def seed_is_complex(seq, shape, reduction, cut):
    return bool(lib().orc_seed_is_complex(_bytes(seq), shape.encode(), reduction, cut))


def shape_packed(seq, pos, shape, reduction):
    key = C.c_uint64()
    ok = lib().orc_shape_packed(_bytes(seq), len(seq), pos, shape.encode(), reduction, C.byref(key))
    return key.value if ok else None


def seed_build(seqs, shape, reduction=0, base=0, cut=0.0):
    letters, off = concat(seqs)
    out = C.POINTER(_Entry)()
    n = C.c_size_t()
    rc = lib().orc_seed_build(letters.ctypes.data_as(C.c_void_p), off.ctypes.data_as(C.c_void_p),
                              C.c_size_t(len(seqs)), shape.encode(), reduction, C.c_uint32(base), C.c_double(cut),
                              C.byref(out), C.byref(n))
    if rc:
        raise ValueError(lib().orc_last_error().decode())
    arr = np.array([(out[i].key, out[i].seq, out[i].pos) for i in range(n.value)],
                   dtype=[("key", "u8"), ("seq", "u4"), ("pos", "u4")])
    lib().orc_free(out)
    return arr


def seed_join(q, r, n_targets, max_expand=4096):
    def to_c(e):
        a = (_Entry * max(len(e), 1))()
        for i, (k, s, p) in enumerate(zip(e["key"], e["seq"], e["pos"])):
            a[i] = _Entry(int(k), int(s), int(p))
        return a
    out = C.POINTER(_Hit)()
    n = C.c_size_t()
    lib().orc_join(to_c(q), C.c_size_t(len(q)), to_c(r), C.c_size_t(len(r)), C.c_size_t(n_targets),
                   C.c_size_t(max_expand), C.byref(out), C.byref(n))
    hits = [(out[i].query, out[i].qpos, out[i].subject, out[i].spos) for i in range(n.value)]
    lib().orc_free(out)
    return hits


def xdrop(q, s, qa, sa, xd=20, matrix="BLOSUM62"):
    o = _Seg()
    lib().orc_xdrop(_bytes(q), C.c_size_t(len(q)), _bytes(s), C.c_size_t(len(s)), C.c_size_t(qa), C.c_size_t(sa),
                    matrix.encode(), xd, C.byref(o))
    return (o.q_start, o.s_start, o.len, o.score)


def extend_span(q, s, d0, d1, matrix="BLOSUM62", go=-1, ge=-1):
    """(score, q_begin, q_end, s_begin, s_end, ident, pos, mism, gapopen, gaps, length, ops) or None; cells."""
    o = _Aligned()
    cap = len(q) + len(s) + 2
    ops = (C.c_uint32 * cap)()
    lib().orc_extend_span(_bytes(q) if len(q) else b"\0", C.c_size_t(len(q)), _bytes(s) if len(s) else b"\0",
                          C.c_size_t(len(s)), C.c_int64(d0), C.c_int64(d1), matrix.encode(), go, ge, C.byref(o),
                          ops, C.c_size_t(cap))
    if not o.found:
        return None, o.cells
    return (o.score, o.q_begin, o.q_end, o.s_begin, o.s_end, o.identities, o.positives, o.mismatches,
            o.gap_openings, o.gaps, o.length, tuple(ops[i] for i in range(o.n_ops))), o.cells


def search(db_seqs, targets, sensitivity="default", evalue=1e-3, max_target_seqs=25, max_hsps=1, index_chunks=None,
           seed_cut=None, threads=1, matrix="BLOSUM62", gap_open=-1, gap_extend=-1, t_query=None, t_frame=None,
           merge=False,
           n_queries=None):
    """search::run (per-target HSP lists) and run counters."""
    dl, do = concat(db_seqs)
    tl, to = concat(targets)
    n_t = len(targets)
    tq = np.ascontiguousarray(np.arange(n_t) if t_query is None else t_query, dtype=np.uint32)
    tf = np.ascontiguousarray(np.zeros(n_t) if t_frame is None else t_frame, dtype=np.uint8)
    cfg = _Cfg(matrix.encode(), gap_open, gap_extend, evalue, max_target_seqs, max_hsps, sensitivity.encode(),
               -1 if index_chunks is None else index_chunks, 0 if seed_cut is None else 1,
               0.0 if seed_cut is None else seed_cut, threads, 0)
    hsps = C.POINTER(_Hsp)()
    n_out = (n_queries if merge else n_t)
    offs = (C.c_uint64 * (max(n_out, n_t) + 1))()
    ops = C.POINTER(C.c_uint32)()
    n_ops = C.c_uint64()
    st = _Stats()
    rc = lib().orc_search(dl.ctypes.data_as(C.c_void_p), do.ctypes.data_as(C.c_void_p), C.c_size_t(len(db_seqs)),
                          C.c_uint64(int(do[-1])), tl.ctypes.data_as(C.c_void_p), to.ctypes.data_as(C.c_void_p),
                          tq.ctypes.data_as(C.c_void_p), tf.ctypes.data_as(C.c_void_p), C.c_size_t(n_t),
                          C.byref(cfg), int(merge), C.c_size_t(n_queries or 0), C.byref(hsps), offs, C.byref(ops),
                          C.byref(n_ops), C.byref(st))
    if rc:
        raise ValueError(lib().orc_last_error().decode())
    lists = []
    for t in range(n_out):
        lst = []
        for k in range(offs[t], offs[t + 1]):
            h = hsps[k]
            o = tuple(ops[h.ops_offset + i] for i in range(h.n_ops))
            lst.append((h.query, h.subject, h.frame, h.score, h.q_begin, h.q_end, h.s_begin, h.s_end, h.bits,
                        h.evalue, h.identities, h.positives, h.mismatches, h.gap_openings, h.gaps, h.length, o))
        lists.append(lst)
    lib().orc_free(hsps)
    lib().orc_free(ops)
    stats = {name: getattr(st, name) for name, _ in _Stats._fields_}
    return lists, stats
