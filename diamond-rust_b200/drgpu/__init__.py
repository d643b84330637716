"""Python binding (ctypes) of the drgpu C ABI (include/drgpu.h).

The library is the product: CUDA kernels for sm_100a behind an ``extern "C"``
interface.  This module only marshals numpy arrays across that boundary; it
has no compute path of its own and raises ``DrgError`` when the shared
library or a CUDA device is missing (there is no CPU fallback).

The entry points mirror the diamond-rust crate: ``seed_build``
(seed::build), ``seed_join`` (seed::join_into), ``xdrop`` (ungapped::xdrop),
``extend_span`` / ``extend_span_scores`` (gapped::extend_span),
``search`` (search::run) and ``merge_frames`` (search::merge_frames).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libdrgpu.so")

DRG_OK = 0
ERRORS = {1: "invalid argument", 2: "out of memory", 3: "CUDA error", 4: "I/O error", 5: "device wait timed out",
          6: "no CUDA device"}


class DrgError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"drgpu error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class SeedEntry(C.Structure):
    _fields_ = [("key", C.c_uint64), ("seq", C.c_uint32), ("pos", C.c_uint32)]


class SeedHit(C.Structure):
    _fields_ = [("query", C.c_uint32), ("qpos", C.c_uint32), ("subject", C.c_uint32), ("spos", C.c_uint32)]


class Segment(C.Structure):
    _fields_ = [("q_start", C.c_uint64), ("s_start", C.c_uint64), ("len", C.c_uint64), ("score", C.c_int32),
                ("pad", C.c_int32)]


class XdropJob(C.Structure):
    _fields_ = [("query", C.c_uint32), ("subject", C.c_uint32), ("qa", C.c_uint64), ("sa", C.c_uint64)]


class SpanJob(C.Structure):
    _fields_ = [("query", C.c_uint32), ("subject", C.c_uint32), ("d0", C.c_int64), ("d1", C.c_int64)]


class Aligned(C.Structure):
    _fields_ = [("found", C.c_int32), ("score", C.c_int32), ("q_begin", C.c_uint64), ("q_end", C.c_uint64),
                ("s_begin", C.c_uint64), ("s_end", C.c_uint64), ("identities", C.c_uint32),
                ("positives", C.c_uint32), ("mismatches", C.c_uint32), ("gap_openings", C.c_uint32),
                ("gaps", C.c_uint32), ("length", C.c_uint32), ("cells", C.c_uint64), ("n_ops", C.c_uint32),
                ("pad", C.c_uint32), ("ops_offset", C.c_uint64)]


class Hsp(C.Structure):
    _fields_ = [("query", C.c_uint32), ("subject", C.c_uint32), ("frame", C.c_uint32), ("score", C.c_int32),
                ("q_begin", C.c_uint32), ("q_end", C.c_uint32), ("s_begin", C.c_uint32), ("s_end", C.c_uint32),
                ("bits", C.c_double), ("evalue", C.c_double), ("identities", C.c_uint32),
                ("positives", C.c_uint32), ("mismatches", C.c_uint32), ("gap_openings", C.c_uint32),
                ("gaps", C.c_uint32), ("length", C.c_uint32), ("ops_offset", C.c_uint64), ("n_ops", C.c_uint32),
                ("pad", C.c_uint32)]


class Tuning(C.Structure):
    _fields_ = [("sw_wide_min_width", C.c_int32), ("sw_min_packed_width", C.c_int32), ("sw_transpose", C.c_int32),
                ("sort_small_tiles", C.c_int32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class SearchConfig(C.Structure):
    _fields_ = [("matrix", C.c_char_p), ("gap_open", C.c_int32), ("gap_extend", C.c_int32), ("evalue", C.c_double),
                ("max_target_seqs", C.c_uint32), ("max_hsps", C.c_uint32), ("sensitivity", C.c_char_p),
                ("index_chunks", C.c_int32), ("has_seed_cut", C.c_int32), ("seed_cut", C.c_double),
                ("threads", C.c_uint32), ("flags", C.c_uint32), ("max_hits_per_pass", C.c_uint64)]


class RunStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("query_seeds", "ref_seeds", "hits", "unique_hits", "xdrops", "segments",
                                          "bands", "bands_computed", "dp_cells_ref", "dp_cells_gpu",
                                          "traced_bands", "hsps")] + \
               [(n, C.c_double) for n in ("ms_total", "ms_seed", "ms_join", "ms_sort", "ms_ungapped", "ms_bands",
                                          "ms_sw", "ms_select", "ms_trace", "ms_host", "ms_h2d", "ms_d2h",
                                          "ms_sw_kernel")] + \
               [("sw_launches", C.c_uint64), ("kernel_launches", C.c_uint64), ("exact_bands", C.c_uint64),
                ("sw_class_tasks", C.c_uint64 * 4), ("sw_class_max_steps", C.c_uint64 * 4),
                ("ms_sw_class", C.c_double * 4), ("ms_trace_kernel", C.c_double), ("dp_cells_lane", C.c_uint64),
                ("sw_wide_bands", C.c_uint64), ("ms_sw_wide", C.c_double), ("dp_cells_issued", C.c_uint64),
                ("index_hits", C.c_uint64), ("sw_transposed_bands", C.c_uint64),
                ("seed_shapes", C.c_uint64), ("query_blocks", C.c_uint64), ("hit_passes", C.c_uint64)]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if isinstance(v, C.Array) else v
        return d


class Result(C.Structure):
    _fields_ = [("hsps", C.POINTER(Hsp)), ("n_hsps", C.c_uint64), ("target_offsets", C.POINTER(C.c_uint64)),
                ("n_targets", C.c_uint64), ("ops", C.POINTER(C.c_uint32)), ("n_ops", C.c_uint64),
                ("stats", RunStats)]


_P = C.POINTER
_u8p = _P(C.c_uint8)
_u32p = _P(C.c_uint32)
_u64p = _P(C.c_uint64)
_i32p = _P(C.c_int32)

# name -> (restype, argtypes)
_SIGNATURES = {
    "drg_ctx_create": (C.c_int, [C.c_int, _P(C.c_void_p)]),
    "drg_ctx_destroy": (None, [C.c_void_p]),
    "drg_last_error": (C.c_char_p, [C.c_void_p]),
    "drg_version": (C.c_char_p, []),
    "drg_free": (None, [C.c_void_p]),
    "drg_seed_build": (C.c_int, [C.c_void_p, _u8p, _u64p, C.c_uint64, C.c_char_p, C.c_int32, C.c_uint32,
                                 C.c_double, _P(_P(SeedEntry)), _u64p]),
    "drg_seed_join": (C.c_int, [C.c_void_p, _P(SeedEntry), C.c_uint64, _P(SeedEntry), C.c_uint64, C.c_uint64,
                                C.c_uint64, _P(_P(SeedHit)), _u64p]),
    "drg_seed_chunks": (C.c_int, [C.c_uint64, C.c_uint64, _u64p, _u64p]),
    "drg_ctx_get_tuning": (C.c_int, [C.c_void_p, _P(Tuning)]),
    "drg_ctx_set_tuning": (C.c_int, [C.c_void_p, _P(Tuning)]),
    "drg_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _P(SearchConfig), C.c_char_p, C.c_int32,
                               _P(Tuning), _P(C.c_double), _P(C.c_double)]),
    "drg_radix_sort": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, _u32p, C.c_uint64, C.c_int32, C.c_int32,
                                 C.c_int32]),
    "drg_xdrop_batch": (C.c_int, [C.c_void_p, _u8p, _u64p, C.c_uint64, _u8p, _u64p, C.c_uint64, _P(XdropJob),
                                  C.c_uint64, C.c_char_p, C.c_int32, _P(Segment)]),
    "drg_extend_span_batch": (C.c_int, [C.c_void_p, _u8p, _u64p, C.c_uint64, _u8p, _u64p, C.c_uint64,
                                        _P(SpanJob), C.c_uint64, C.c_char_p, C.c_int32, C.c_int32, _P(Aligned),
                                        _P(_u32p), _u64p]),
    "drg_extend_span_scores": (C.c_int, [C.c_void_p, _u8p, _u64p, C.c_uint64, _u8p, _u64p, C.c_uint64,
                                         _P(SpanJob), C.c_uint64, C.c_char_p, C.c_int32, C.c_int32, _i32p,
                                         _P(RunStats)]),
    "drg_extend_span_noalloc": (C.c_int, [C.c_void_p, _u64p, C.c_uint64, C.c_void_p, _u64p, C.c_uint64,
                                          _P(SpanJob), C.c_uint64, C.c_char_p, C.c_int32, C.c_int32, C.c_void_p,
                                          C.c_void_p, C.c_uint64, C.c_void_p, C.c_char_p, C.c_size_t]),
    "drg_db_create": (C.c_int, [C.c_void_p, _u8p, _u64p, C.c_uint64, _P(C.c_void_p)]),
    "drg_db_destroy": (None, [C.c_void_p]),
    "drg_db_set_index_budget": (C.c_int, [C.c_void_p, C.c_uint64]),
    "drg_batch_create_blastx": (C.c_int, [C.c_void_p, _u8p, _u64p, C.c_uint64, C.c_int64, _P(C.c_void_p)]),
    "drg_translate_reads": (C.c_int, [C.c_void_p, _u8p, _u64p, C.c_uint64, C.c_int64, _P(_P(C.c_uint8)),
                                      _P(_P(C.c_uint64)), _P(_P(C.c_uint32)), _P(_P(C.c_uint8)), _P(C.c_uint64)]),
    "drg_batch_targets": (C.c_int, [C.c_void_p, _P(C.c_uint64), C.c_void_p, C.c_void_p]),
    "drg_db_index_stats": (C.c_int, [C.c_void_p, C.c_void_p]),
    "drg_batch_create": (C.c_int, [C.c_void_p, _u8p, _u64p, _u32p, _u8p, C.c_uint64, _P(C.c_void_p)]),
    "drg_batch_create_requests": (C.c_int, [C.c_void_p, _u8p, _u64p, _u32p, _u8p, _u32p, C.c_uint64,
                                            _P(C.c_void_p)]),
    "drg_batch_destroy": (None, [C.c_void_p]),
    "drg_search_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _P(SearchConfig), _P(Result)]),
    "drg_search_run": (C.c_int, [C.c_void_p, _u8p, _u64p, C.c_uint64, _u8p, _u64p, _u32p, _u8p, C.c_uint64,
                                 _P(SearchConfig), _P(Result)]),
    "drg_search_run_per_stage": (C.c_int, [C.c_void_p, _u8p, _u64p, C.c_uint64, _u8p, _u64p, _u32p, _u8p,
                                           C.c_uint64, _P(SearchConfig), _P(Result)]),
    "drg_merge_frames": (C.c_int, [_P(Result), C.c_uint64, _u32p, C.c_uint64, C.c_uint64]),
    "drg_result_free": (None, [_P(Result)]),
    "drg_matrix_evalue": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_uint64,
                                    C.c_uint64, _P(C.c_double), _P(C.c_double)]),
    "drg_probe_int_peak": (C.c_int, [C.c_void_p, _P(C.c_double), _P(C.c_double)]),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libdrgpu.so and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise DrgError(6, f"{path} is missing: build it with `make -C diamond-rust_b200` (no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def _u8(a):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    return a, _ptr(a, C.c_uint8)


def _u64(a):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a, _ptr(a, C.c_uint64)


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, _ptr(a, C.c_uint32)


def offsets_of(seqs) -> np.ndarray:
    off = np.zeros(len(seqs) + 1, dtype=np.uint64)
    if len(seqs):
        off[1:] = np.cumsum([len(s) for s in seqs])
    return off


def concat(seqs) -> tuple[np.ndarray, np.ndarray]:
    """List of uint8 letter arrays -> (letters, offsets)."""
    off = offsets_of(seqs)
    letters = np.concatenate([np.asarray(s, dtype=np.uint8) for s in seqs]) if len(seqs) else np.zeros(0, np.uint8)
    return np.ascontiguousarray(letters, dtype=np.uint8), off


@dataclass
class HspRecord:
    query: int
    subject: int
    frame: int
    score: int
    q_begin: int
    q_end: int
    s_begin: int
    s_end: int
    bits: float
    evalue: float
    identities: int
    positives: int
    mismatches: int
    gap_openings: int
    gaps: int
    length: int
    ops: tuple

    def key(self):
        return (self.query, self.subject, self.frame, self.score, self.q_begin, self.q_end, self.s_begin, self.s_end,
                self.bits, self.evalue, self.identities, self.positives, self.mismatches, self.gap_openings,
                self.gaps, self.length, self.ops)


class ResultArrays:
    """A result copied out of the library in three bulk copies: hsps (numpy
    structured array of drg_hsp), target_offsets (n_targets + 1) and ops.
    lists() builds the per-target HspRecord lists on demand."""

    def __init__(self, res: Result):
        n, n_t = int(res.n_hsps), int(res.n_targets)
        self.hsps = np.ctypeslib.as_array(res.hsps, shape=(n,)).copy() if n else np.zeros(0, _HSP_DTYPE)
        self.target_offsets = (np.ctypeslib.as_array(res.target_offsets, shape=(n_t + 1,)).copy() if n_t
                               else np.zeros(1, np.uint64))
        self.ops = (np.ctypeslib.as_array(res.ops, shape=(int(res.n_ops),)).copy() if res.n_ops
                    else np.zeros(0, np.uint32))

    def lists(self, query_shift=0):
        out = []
        h, offs, ops = self.hsps, self.target_offsets.tolist(), self.ops
        cols = [h[f].tolist() for f in ("query", "subject", "frame", "score", "q_begin", "q_end", "s_begin", "s_end",
                                        "bits", "evalue", "identities", "positives", "mismatches", "gap_openings",
                                        "gaps", "length", "ops_offset", "n_ops")]
        for t in range(len(offs) - 1):
            lst = []
            for k in range(offs[t], offs[t + 1]):
                o, n = cols[16][k], cols[17][k]
                lst.append(HspRecord(cols[0][k] - query_shift, *(c[k] for c in cols[1:16]),
                                     tuple(ops[o:o + n].tolist())))
            out.append(lst)
        return out


_HSP_DTYPE = np.ctypeslib.as_array((Hsp * 1)()).dtype


def _result_lists(res: Result):
    return ResultArrays(res).lists()


def make_config(sensitivity="default", matrix="BLOSUM62", gap_open=-1, gap_extend=-1, evalue=1e-3,
                max_target_seqs=25, max_hsps=1, index_chunks=None, seed_cut=None, threads=0,
                max_hits_per_pass=0) -> SearchConfig:
    c = SearchConfig()
    c.matrix = matrix.encode()
    c.gap_open = gap_open
    c.gap_extend = gap_extend
    c.evalue = evalue
    c.max_target_seqs = max_target_seqs
    c.max_hsps = max_hsps
    c.sensitivity = sensitivity.encode()
    c.index_chunks = -1 if index_chunks is None else int(index_chunks)
    c.has_seed_cut = 0 if seed_cut is None else 1
    c.seed_cut = 0.0 if seed_cut is None else float(seed_cut)
    c.threads = threads
    c.flags = 0
    c.max_hits_per_pass = max_hits_per_pass
    return c


class Context:
    """One device context (CUDA stream + cached device buffers)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.drg_ctx_create(device, C.byref(h))
        if rc != DRG_OK:
            raise DrgError(rc, "cannot create a device context")
        self.h = h

    def close(self):
        if self.h:
            self.lib.drg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != DRG_OK:
            raise DrgError(rc, self.lib.drg_last_error(self.h).decode())

    # ---- stage entry points -------------------------------------------------
    def seed_build(self, seqs, shape_code: str, reduction: int = 0, base: int = 0, cut: float = 0.0):
        letters, off = concat(seqs)
        la, lp = _u8(letters if len(letters) else np.zeros(1, np.uint8))
        oa, op = _u64(off)
        out = C.POINTER(SeedEntry)()
        n = C.c_uint64()
        self._check(self.lib.drg_seed_build(self.h, lp, op, len(seqs), shape_code.encode(), reduction, base, cut,
                                            C.byref(out), C.byref(n)))
        arr = np.array([(out[i].key, out[i].seq, out[i].pos) for i in range(n.value)],
                       dtype=[("key", "u8"), ("seq", "u4"), ("pos", "u4")])
        self.lib.drg_free(out)
        return arr

    def tuning(self):
        t = Tuning()
        self._check(self.lib.drg_ctx_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        t = Tuning()
        self._check(self.lib.drg_ctx_get_tuning(self.h, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, int(v))
        self._check(self.lib.drg_ctx_set_tuning(self.h, C.byref(t)))

    def autotune(self, db, batch, config, cache_path=None, reps=2):
        """drg_autotune: the best tuning for (db, batch, config), left in the
        context; returns (tuning, ms under the starting tuning, ms best)."""
        t, a, b = Tuning(), C.c_double(), C.c_double()
        self._check(self.lib.drg_autotune(self.h, db.h, batch.h, C.byref(config),
                                          None if cache_path is None else cache_path.encode(), reps, C.byref(t),
                                          C.byref(a), C.byref(b)))
        return t.as_dict(), a.value, b.value

    def radix_sort(self, keys, vals=None, begin_bit=0, end_bit=None, count_on_device=False):
        """The device radix sort (stable) of u32 or u64 keys, with optional
        u32 values; returns sorted copies."""
        k = np.ascontiguousarray(keys).copy()
        if k.dtype not in (np.uint32, np.uint64):
            raise TypeError("keys must be uint32 or uint64")
        v = None if vals is None else np.ascontiguousarray(vals, dtype=np.uint32).copy()
        kb = k.dtype.itemsize
        eb = 8 * kb if end_bit is None else end_bit
        self._check(self.lib.drg_radix_sort(self.h, k.ctypes.data_as(C.c_void_p), kb,
                                            None if v is None else v.ctypes.data_as(_u32p), len(k), begin_bit, eb,
                                            int(count_on_device)))
        return k, v

    def seed_join(self, q_entries, r_entries, n_targets: int, max_expand: int = 4096):
        def to_c(e):
            a = (SeedEntry * max(len(e), 1))()
            for i, (k, s, p) in enumerate(zip(e["key"], e["seq"], e["pos"])):
                a[i] = SeedEntry(int(k), int(s), int(p))
            return a
        qa, ra = to_c(q_entries), to_c(r_entries)
        out = C.POINTER(SeedHit)()
        n = C.c_uint64()
        self._check(self.lib.drg_seed_join(self.h, qa, len(q_entries), ra, len(r_entries), n_targets, max_expand,
                                           C.byref(out), C.byref(n)))
        hits = [(out[i].query, out[i].qpos, out[i].subject, out[i].spos) for i in range(n.value)]
        self.lib.drg_free(out)
        return hits

    def xdrop(self, queries, subjects, jobs, matrix="BLOSUM62", xdrop=20):
        ql, qo = concat(queries)
        sl, so = concat(subjects)
        ql = ql if len(ql) else np.zeros(1, np.uint8)
        sl = sl if len(sl) else np.zeros(1, np.uint8)
        ja = (XdropJob * max(len(jobs), 1))(*[XdropJob(*j) for j in jobs])
        out = (Segment * max(len(jobs), 1))()
        self._check(self.lib.drg_xdrop_batch(self.h, _ptr(ql, C.c_uint8), _ptr(qo, C.c_uint64), len(queries),
                                             _ptr(sl, C.c_uint8), _ptr(so, C.c_uint64), len(subjects), ja,
                                             len(jobs), matrix.encode(), xdrop, out))
        return [(out[i].q_start, out[i].s_start, out[i].len, out[i].score) for i in range(len(jobs))]

    def extend_span(self, queries, subjects, jobs, matrix="BLOSUM62", gap_open=-1, gap_extend=-1):
        """Full gapped::extend_span (score, coordinates, stats, ops) per job; None when no alignment."""
        ql, qo = concat(queries)
        sl, so = concat(subjects)
        ql = ql if len(ql) else np.zeros(1, np.uint8)
        sl = sl if len(sl) else np.zeros(1, np.uint8)
        ja = (SpanJob * max(len(jobs), 1))(*[SpanJob(*j) for j in jobs])
        out = (Aligned * max(len(jobs), 1))()
        ops = C.POINTER(C.c_uint32)()
        nops = C.c_uint64()
        self._check(self.lib.drg_extend_span_batch(self.h, _ptr(ql, C.c_uint8), _ptr(qo, C.c_uint64), len(queries),
                                                   _ptr(sl, C.c_uint8), _ptr(so, C.c_uint64), len(subjects), ja,
                                                   len(jobs), matrix.encode(), gap_open, gap_extend, out,
                                                   C.byref(ops), C.byref(nops)))
        res = []
        for i in range(len(jobs)):
            a = out[i]
            if not a.found:
                res.append(None)
                continue
            o = tuple(ops[a.ops_offset + k] for k in range(a.n_ops))
            res.append((a.score, a.q_begin, a.q_end, a.s_begin, a.s_end, a.identities, a.positives, a.mismatches,
                        a.gap_openings, a.gaps, a.length, o))
        self.lib.drg_free(ops)
        return res

    def extend_span_scores(self, queries, subjects, jobs, matrix="BLOSUM62", gap_open=-1, gap_extend=-1):
        """Band scores through the packed score kernel (0 = None) and run stats."""
        ql, qo = concat(queries)
        sl, so = concat(subjects)
        ql = ql if len(ql) else np.zeros(1, np.uint8)
        sl = sl if len(sl) else np.zeros(1, np.uint8)
        ja = (SpanJob * max(len(jobs), 1))(*[SpanJob(*j) for j in jobs])
        scores = np.zeros(max(len(jobs), 1), dtype=np.int32)
        st = RunStats()
        self._check(self.lib.drg_extend_span_scores(self.h, _ptr(ql, C.c_uint8), _ptr(qo, C.c_uint64),
                                                    len(queries), _ptr(sl, C.c_uint8), _ptr(so, C.c_uint64),
                                                    len(subjects), ja, len(jobs), matrix.encode(), gap_open,
                                                    gap_extend, _ptr(scores, C.c_int32), C.byref(st)))
        return scores[:len(jobs)], st.as_dict()

    # ---- whole path ----------------------------------------------------------
    def search(self, db_letters, db_offsets, t_letters, t_offsets, config: SearchConfig, t_query=None, t_frame=None):
        """search::run from host buffers (uploads, searches, downloads)."""
        dl, dlp = _u8(db_letters if len(db_letters) else np.zeros(1, np.uint8))
        do, dop = _u64(db_offsets)
        tl, tlp = _u8(t_letters if len(t_letters) else np.zeros(1, np.uint8))
        to, top = _u64(t_offsets)
        n_t = len(t_offsets) - 1
        tq, tqp = _u32(np.arange(n_t) if t_query is None else t_query)
        tf, tfp = _u8(np.zeros(n_t) if t_frame is None else t_frame)
        res = Result()
        self._check(self.lib.drg_search_run(self.h, dlp, dop, len(db_offsets) - 1, tlp, top, tqp, tfp, n_t,
                                            C.byref(config), C.byref(res)))
        try:
            return _result_lists(res), res.stats.as_dict()
        finally:
            self.lib.drg_result_free(C.byref(res))

    def search_per_stage(self, db_letters, db_offsets, t_letters, t_offsets, config: SearchConfig, t_query=None,
                         t_frame=None, want_lists=True):
        """search::run orchestrated on the host over the per-stage entry
        points (drg_search_run_per_stage): the plain per-stage drop-in."""
        dl, dlp = _u8(db_letters if len(db_letters) else np.zeros(1, np.uint8))
        do, dop = _u64(db_offsets)
        tl, tlp = _u8(t_letters if len(t_letters) else np.zeros(1, np.uint8))
        to, top = _u64(t_offsets)
        n_t = len(t_offsets) - 1
        tq, tqp = _u32(np.arange(n_t) if t_query is None else t_query)
        tf, tfp = _u8(np.zeros(n_t) if t_frame is None else t_frame)
        res = Result()
        self._check(self.lib.drg_search_run_per_stage(self.h, dlp, dop, len(db_offsets) - 1, tlp, top, tqp, tfp,
                                                      n_t, C.byref(config), C.byref(res)))
        try:
            return (_result_lists(res) if want_lists else None), res.stats.as_dict(), int(res.n_hsps)
        finally:
            self.lib.drg_result_free(C.byref(res))

    def search_counts(self, db_letters, db_offsets, t_letters, t_offsets, config: SearchConfig):
        """The same C-ABI call as ``search``, returning only (n_hsps, n_ops, stats): for timing the
        drop-in call without building Python records."""
        dl, dlp = _u8(db_letters if len(db_letters) else np.zeros(1, np.uint8))
        do, dop = _u64(db_offsets)
        tl, tlp = _u8(t_letters if len(t_letters) else np.zeros(1, np.uint8))
        to, top = _u64(t_offsets)
        n_t = len(t_offsets) - 1
        tq, tqp = _u32(np.arange(n_t))
        tf, tfp = _u8(np.zeros(n_t))
        res = Result()
        self._check(self.lib.drg_search_run(self.h, dlp, dop, len(db_offsets) - 1, tlp, top, tqp, tfp, n_t,
                                            C.byref(config), C.byref(res)))
        n_hsps, n_ops = int(res.n_hsps), int(res.n_ops)
        stats = res.stats.as_dict()
        self.lib.drg_result_free(C.byref(res))
        return n_hsps, n_ops, stats

    def translate_reads(self, reads, min_orf=-1):
        """blastx front end on the device: the kept frames of each read as
        (list of letter arrays, read index per frame, frame 0-5 per frame)."""
        nl, no = _reads_buffers(reads)
        nlp, nop = _ptr(nl, C.c_uint8), _ptr(no, C.c_uint64)
        L, O, Q, F = (C.POINTER(C.c_uint8)(), C.POINTER(C.c_uint64)(), C.POINTER(C.c_uint32)(),
                      C.POINTER(C.c_uint8)())
        n = C.c_uint64()
        self._check(self.lib.drg_translate_reads(self.h, nlp, nop, len(no) - 1, int(min_orf), C.byref(L),
                                                 C.byref(O), C.byref(Q), C.byref(F), C.byref(n)))
        try:
            k = n.value
            offs = np.ctypeslib.as_array(O, shape=(k + 1,)).copy()
            total = int(offs[-1])
            letters = np.ctypeslib.as_array(L, shape=(max(total, 1),))[:total].copy()
            query = np.ctypeslib.as_array(Q, shape=(max(k, 1),))[:k].copy()
            frame = np.ctypeslib.as_array(F, shape=(max(k, 1),))[:k].copy()
        finally:
            for p in (L, O, Q, F):
                self.lib.drg_free(C.cast(p, C.c_void_p))
        frames = [letters[offs[i]:offs[i + 1]] for i in range(k)]
        return frames, query, frame

    def probe_int_peak(self):
        ops, mhz = C.c_double(), C.c_double()
        self._check(self.lib.drg_probe_int_peak(self.h, C.byref(ops), C.byref(mhz)))
        return ops.value, mhz.value


class IndexStats(C.Structure):
    _fields_ = [("entries", C.c_uint64), ("bytes", C.c_uint64), ("hits", C.c_uint64), ("misses", C.c_uint64),
                ("evictions", C.c_uint64)]


class ResidentDb:
    """Database letters resident in device memory (drg_db).

    index_budget > 0 keeps the sorted reference seeds of each preset and index
    chunk in device memory for later searches (drg_db_set_index_budget)."""

    def __init__(self, ctx: Context, letters, offsets, index_budget=0):
        self.ctx = ctx
        self._l, lp = _u8(letters if len(letters) else np.zeros(1, np.uint8))
        self._o, op = _u64(offsets)
        h = C.c_void_p()
        ctx._check(ctx.lib.drg_db_create(ctx.h, lp, op, len(offsets) - 1, C.byref(h)))
        self.h = h
        if index_budget:
            self.set_index_budget(index_budget)

    def set_index_budget(self, nbytes):
        self.ctx._check(self.ctx.lib.drg_db_set_index_budget(self.h, int(nbytes)))

    def index_stats(self):
        s = IndexStats()
        self.ctx._check(self.ctx.lib.drg_db_index_stats(self.h, C.byref(s)))
        return {k: int(getattr(s, k)) for k, _ in IndexStats._fields_}

    def close(self):
        if self.h:
            self.ctx.lib.drg_db_destroy(self.h)
            self.h = None


class ResidentBatch:
    """Query batch resident in device memory (drg_batch)."""

    def __init__(self, ctx: Context, letters, offsets, query=None, frame=None, request=None):
        """request[t]: request id of target t; each request is searched as if alone."""
        self.ctx = ctx
        n = len(offsets) - 1
        self._l, lp = _u8(letters if len(letters) else np.zeros(1, np.uint8))
        self._o, op = _u64(offsets)
        self._q, qp = _u32(np.arange(n) if query is None else query)
        self._f, fp = _u8(np.zeros(n) if frame is None else frame)
        h = C.c_void_p()
        if request is None:
            ctx._check(ctx.lib.drg_batch_create(ctx.h, lp, op, qp, fp, n, C.byref(h)))
        else:
            self._r, rp = _u32(request)
            ctx._check(ctx.lib.drg_batch_create_requests(ctx.h, lp, op, qp, fp, rp, n, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.ctx.lib.drg_batch_destroy(self.h)
            self.h = None


def _reads_buffers(reads):
    """Nucleotide reads (str or bytes) as one byte buffer with offsets."""
    raw = [r.encode() if isinstance(r, str) else bytes(r) for r in reads]
    offs = np.zeros(len(raw) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in raw]) if raw else []
    buf = np.frombuffer(b"".join(raw) + b"\0", dtype=np.uint8).copy()
    return buf, offs


def blastx_batch(ctx: Context, reads, min_orf=-1):
    """The reads' kept frames, translated on the device, as a resident batch
    (drg_batch_create_blastx); .query / .frame hold each target's read and frame."""
    nl, no = _reads_buffers(reads)
    h = C.c_void_p()
    ctx._check(ctx.lib.drg_batch_create_blastx(ctx.h, _ptr(nl, C.c_uint8), _ptr(no, C.c_uint64), len(no) - 1,
                                               int(min_orf), C.byref(h)))
    b = ResidentBatch.__new__(ResidentBatch)
    b.ctx, b.h = ctx, h
    n = C.c_uint64()
    ctx._check(ctx.lib.drg_batch_targets(h, C.byref(n), None, None))
    b.query = np.zeros(max(n.value, 1), np.uint32)
    b.frame = np.zeros(max(n.value, 1), np.uint8)
    ctx._check(ctx.lib.drg_batch_targets(h, C.byref(n), b.query.ctypes.data_as(C.c_void_p),
                                         b.frame.ctypes.data_as(C.c_void_p)))
    b.query, b.frame = b.query[:n.value], b.frame[:n.value]
    return b


def search_resident(ctx: Context, db: ResidentDb, batch: ResidentBatch, config: SearchConfig, want_lists=True,
                    merge_queries=None):
    """merge_queries = n: the frames' lists merged per query (drg_merge_frames,
    search::merge_frames), by the batch's query index of each target."""
    res = Result()
    ctx._check(ctx.lib.drg_search_batch(ctx.h, db.h, batch.h, C.byref(config), C.byref(res)))
    try:
        if merge_queries is not None:
            tq = np.ascontiguousarray(batch.query, dtype=np.uint32)
            ctx._check(ctx.lib.drg_merge_frames(C.byref(res), merge_queries, _ptr(tq, C.c_uint32), config.max_hsps,
                                                config.max_target_seqs))
        lists = _result_lists(res) if want_lists else None
        return lists, res.stats.as_dict(), int(res.n_hsps)
    finally:
        ctx.lib.drg_result_free(C.byref(res))


def matrix_evalue(raw, qlen, slen, db_letters, matrix="BLOSUM62", gap_open=-1, gap_extend=-1):
    lib = load_library()
    e, b = C.c_double(), C.c_double()
    rc = lib.drg_matrix_evalue(matrix.encode(), gap_open, gap_extend, raw, qlen, slen, db_letters, C.byref(e),
                               C.byref(b))
    if rc != DRG_OK:
        raise DrgError(rc, "matrix")
    return e.value, b.value


def exported_symbols():
    return list(_SIGNATURES)
