"""The allocation-free extend_span entry point (drg_extend_span_noalloc).

Callers that cannot allocate device memory -- services whose own pool owns
every device byte and forbids library allocations on the request path,
real-time loops that may not take allocator locks -- use this entry point with
buffers they already own.  This test is that caller: it owns the device
buffers (through torch) and checks that calls in a row give exactly what the
allocating entry point drg_extend_span_batch gives (exact integer results,
tolerance 0).  It lives in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import drgpu  # noqa: E402
from drgpu import synth  # noqa: E402


def _bind():
    lib = drgpu.load_library()
    fn = lib.drg_extend_span_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.c_uint64, C.c_void_p, C.POINTER(C.c_uint64), C.c_uint64,
                   C.POINTER(drgpu.SpanJob), C.c_uint64, C.c_char_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                   C.c_uint64, C.c_void_p, C.c_char_p, C.c_size_t]
    return fn


def _cases(seed, n_cases, max_len=300, halves=(5, 12, 30, 64)):
    r = np.random.Generator(np.random.PCG64(seed))
    queries, subjects, jobs = [], [], []
    for i in range(n_cases):
        q = synth.random_protein(r, int(r.integers(1, max_len)))
        s = synth.mutate(r, q, float(r.uniform(0.3, 0.9))) if i % 2 else synth.random_protein(r, int(r.integers(1, max_len)))
        if len(s) == 0:
            s = synth.random_protein(r, 5)
        d = int(r.integers(-len(s) + 1, len(q)))
        half = int(r.choice(halves))
        queries.append(q)
        subjects.append(s)
        jobs.append((i, i, d - half, d + half))
    return queries, subjects, jobs


def _noalloc(fn, queries, subjects, jobs):
    import torch
    ql, qo = drgpu.concat(queries)
    sl, so = drgpu.concat(subjects)
    dq = torch.from_numpy(ql).cuda()
    ds = torch.from_numpy(sl).cuda()
    cap = int(sum(len(queries[j[0]]) + len(subjects[j[1]]) for j in jobs))
    out = torch.zeros(len(jobs) * C.sizeof(drgpu.Aligned), dtype=torch.uint8, device="cuda")
    ops = torch.zeros(max(cap, 1), dtype=torch.int32, device="cuda")
    ja = (drgpu.SpanJob * len(jobs))(*[drgpu.SpanJob(*j) for j in jobs])
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(dq.data_ptr(), qo.ctypes.data_as(C.POINTER(C.c_uint64)), len(queries), ds.data_ptr(),
            so.ctypes.data_as(C.POINTER(C.c_uint64)), len(subjects), ja, len(jobs), b"BLOSUM62", -1, -1,
            out.data_ptr(), ops.data_ptr(), cap, stream, err, 256)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    raw = out.cpu().numpy().tobytes()
    ops_h = ops.cpu().numpy().view(np.uint32)
    res = []
    for i in range(len(jobs)):
        a = drgpu.Aligned.from_buffer_copy(raw, i * C.sizeof(drgpu.Aligned))
        if not a.found:
            res.append(None)
            continue
        o = tuple(int(x) for x in ops_h[a.ops_offset:a.ops_offset + a.n_ops])
        res.append((a.score, a.q_begin, a.q_end, a.s_begin, a.s_end, a.identities, a.positives, a.mismatches,
                    a.gap_openings, a.gaps, a.length, o))
    return res


def test_noalloc_matches_extend_span_batch_twice():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    fn = _bind()
    ctx = drgpu.Context(0)
    try:
        # calls in a row share the static scratch; the last has several jobs
        # per thread of the one-block offset scan (1,024 threads)
        for seed, n, mx, halves in ((101, 120, 300, (5, 12, 30, 64)), (102, 120, 300, (5, 12, 30, 64)),
                                    (103, 2600, 60, (3, 8, 12))):
            queries, subjects, jobs = _cases(seed, n, mx, halves)
            got = _noalloc(fn, queries, subjects, jobs)
            exp = ctx.extend_span(queries, subjects, jobs)
            assert got == exp
            assert any(x is not None for x in got)
    finally:
        ctx.close()


def test_noalloc_rejects_oversized_calls():
    torch = pytest.importorskip("torch")
    fn = _bind()
    q = np.full(5000, 3, np.uint8)
    s = np.full(5000, 3, np.uint8)
    jobs = [(0, 0, -2000, 2000)] * 8  # about 8 x 20 MB of trace: beyond the 32 MiB scratch
    ql, qo = drgpu.concat([q])
    sl, so = drgpu.concat([s])
    dq = torch.from_numpy(ql).cuda()
    out = torch.zeros(len(jobs) * C.sizeof(drgpu.Aligned), dtype=torch.uint8, device="cuda")
    ops = torch.zeros(len(jobs) * 10000, dtype=torch.int32, device="cuda")
    ja = (drgpu.SpanJob * len(jobs))(*[drgpu.SpanJob(*j) for j in jobs])
    err = C.create_string_buffer(256)
    rc = fn(dq.data_ptr(), qo.ctypes.data_as(C.POINTER(C.c_uint64)), 1, dq.data_ptr(),
            so.ctypes.data_as(C.POINTER(C.c_uint64)), 1, ja, len(jobs), b"BLOSUM62", -1, -1, out.data_ptr(),
            ops.data_ptr(), len(jobs) * 10000, torch.cuda.current_stream().cuda_stream, err, 256)
    assert rc == 1
    assert b"static scratch" in err.value


def test_noalloc_rejects_decreasing_offsets():
    torch = pytest.importorskip("torch")
    fn = _bind()
    ql = np.full(64, 3, np.uint8)
    qo = np.array([0, 40, 20, 64], np.uint64)  # sequence 1 would have a negative length
    dq = torch.from_numpy(ql).cuda()
    out = torch.zeros(C.sizeof(drgpu.Aligned), dtype=torch.uint8, device="cuda")
    ops = torch.zeros(256, dtype=torch.int32, device="cuda")
    ja = (drgpu.SpanJob * 1)(drgpu.SpanJob(1, 0, -3, 3))
    err = C.create_string_buffer(256)
    rc = fn(dq.data_ptr(), qo.ctypes.data_as(C.POINTER(C.c_uint64)), 3, dq.data_ptr(),
            qo.ctypes.data_as(C.POINTER(C.c_uint64)), 3, ja, 1, b"BLOSUM62", -1, -1, out.data_ptr(),
            ops.data_ptr(), 256, torch.cuda.current_stream().cuda_stream, err, 256)
    assert rc == 1
    assert b"offsets decrease" in err.value
