"""Serving: a request loop over a database resident in HBM.

Requests (a list of protein queries plus a sensitivity preset) arrive at any
time.  Worker threads, one CUDA context each, share the resident database;
whenever a worker is free it admits every queued request with the preset of
the oldest one, up to a budget of query letters, as one batch
(drg_batch_create_requests) and searches it.  The batch's join cap is counted
per request, so each request's HSP lists equal those of the request searched
alone; requests that arrive while a batch runs wait only for the next free
worker (continuous batching).

The workers' searches take turns on the GPU (one search at a time, in the
order the workers reached the GPU): a search fills the GPU by itself, and two
searches side by side each take about twice as long, which lengthens the tail
of the latency.  What a worker does on the host (assembling the next batch's
letters, building Python records of the last one) overlaps the other worker's
search.  On request (overlap_backlog) the searches overlap under a backlog
instead: each fills the GPU while the other waits on the host.  That raised
the capacity with every request queued (43-46K against 43K queries/s) but,
in a burst of a 20 requests/s stream, held p99 near 1 s: it is off by
default.

Admission protects the oldest request: a batch holds at most max(64k
letters, the oldest request's letters) (merge_floor, merge_ratio), so small
requests share a batch while a large request runs alone and is not delayed by
the work of requests behind it.  (With a plain letter budget of 1M letters,
large requests of one preset merged, and the tail of the latency grew with
the merged batches' work.)  The letter budget caps any batch.
Results come back to the host as three bulk copies per batch (HSP records,
per-target offsets, alignment ops); Python records are built only when a
request's results are read, outside the worker loop.

The plain path (`workers=1, batch=False`) serves one request at a time.
Latency is the wall time from a request's arrival to its results being back on
the host; throughput is queries over the whole run.
"""
from __future__ import annotations

import ctypes as C
import statistics
import threading
import time
from dataclasses import dataclass

import numpy as np

from . import Context, ResidentBatch, ResidentDb, Result, ResultArrays, concat, make_config


@dataclass
class Request:
    rid: int
    preset: str
    queries: list
    arrival: float = 0.0          # seconds, on the server's clock
    done: float = 0.0
    batch_size: int = 0           # requests in the batch that served it
    raw: object = None            # (ResultArrays of the batch, first target, targets)

    @property
    def results(self):
        """Per query: HSP records, query indices within the request."""
        if self.raw is None:
            return []
        arrays, t0, n = self.raw
        offs = arrays.target_offsets
        sub = ResultArrays.__new__(ResultArrays)
        sub.hsps = arrays.hsps[offs[t0]:offs[t0 + n]]
        sub.target_offsets = offs[t0:t0 + n + 1] - offs[t0]
        sub.ops = arrays.ops
        return sub.lists(query_shift=t0)


def batch_arrays(requests):
    """The letters, offsets and request ids of several requests' queries, in
    request order (host work, no GPU)."""
    seqs, rid = [], []
    for k, r in enumerate(requests):
        seqs.extend(r.queries)
        rid.extend([k] * len(r.queries))
    letters, offsets = concat(seqs)
    return letters, offsets, np.asarray(rid, np.uint32)


def search_batch(ctx: Context, db: ResidentDb, requests, preset: str, index_chunks=None, arrays=None,
                 gpu_turn=None):
    """Search several requests of one preset as one batch; each request gets
    its slice of the batch's results (copied to the host in bulk).  `arrays`
    (from batch_arrays) may be built ahead; `gpu_turn`, a lock, is held while
    the batch is on the GPU (upload, search, results, release)."""
    letters, offsets, rid = arrays if arrays is not None else batch_arrays(requests)
    cfg = make_config(sensitivity=preset, index_chunks=index_chunks)
    res = Result()
    turn = gpu_turn if gpu_turn is not None else _NoLock()
    with turn:
        batch = ResidentBatch(ctx, letters, offsets, request=rid)
        try:
            ctx._check(ctx.lib.drg_search_batch(ctx.h, db.h, batch.h, C.byref(cfg), C.byref(res)))
            arrays = ResultArrays(res)
        finally:
            ctx.lib.drg_result_free(C.byref(res))
            batch.close()
    t = 0
    for r in requests:
        n = len(r.queries)
        r.raw = (arrays, t, n)
        r.batch_size = len(requests)
        t += n
    return requests


class _NoLock:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


class Server:
    """Continuous-batching request loop over one resident database."""

    def __init__(self, db_letters, db_offsets, workers=2, batch=True, budget_letters=1_000_000, device=0,
                 index_chunks=None, index_budget=0, merge_ratio=1.0, merge_floor=64_000, tune_cache=None,
                 overlap_backlog=None):
        self.ctxs = [Context(device) for _ in range(workers)]
        # index_budget > 0: each preset's sorted reference seeds stay resident
        self.db = ResidentDb(self.ctxs[0], db_letters, db_offsets, index_budget=index_budget)
        self.batch = batch
        self.budget = budget_letters
        # a batch holds at most max(merge_floor, merge_ratio x its oldest
        # request's letters) (and the budget): later requests merged into a
        # large request delay it by their work, small ones barely
        self.merge_ratio = merge_ratio
        self.merge_floor = merge_floor
        # tune_cache (a file path): warm() autotunes each preset on its warm-up
        # request (drg_autotune, results cached in the file) and each batch of
        # that preset runs with its tuning; no tuning changes any result
        self.tune_cache = tune_cache
        self.tunings: dict = {}
        self.base_tuning = self.ctxs[0].tuning()
        # overlap_backlog = n: with n or more requests still queued behind a
        # batch, the batch does not wait for its turn, and the searches overlap
        # on the GPU, filling each other's host phases (more throughput under
        # a backlog, at the price of the tail: off by default)
        self.overlap_backlog = overlap_backlog
        self.index_chunks = index_chunks
        self.pending: list[Request] = []
        self.lock = threading.Condition()
        self.gpu_turn = threading.Lock()  # one search on the GPU at a time
        self.closed = False
        self.finished: list[Request] = []
        self.t0 = time.perf_counter()
        self.errors: list[BaseException] = []
        self.threads = [threading.Thread(target=self._worker, args=(c,), daemon=True) for c in self.ctxs]
        for t in self.threads:
            t.start()

    def now(self):
        return time.perf_counter() - self.t0

    def submit(self, req: Request):
        with self.lock:
            req.arrival = self.now()
            self.pending.append(req)
            self.lock.notify()

    def _take(self):
        """The oldest request and, when batching, every queued request of its
        preset that fits the letter budget (admission by memory)."""
        head = self.pending[0]
        if not self.batch:
            self.pending.pop(0)
            return [head]
        take, used = [], 0
        cap = self.budget
        if self.merge_ratio is not None:
            head_size = sum(len(q) for q in head.queries)
            cap = min(cap, max(self.merge_floor, self.merge_ratio * head_size))
        for r in list(self.pending):
            if r.preset != head.preset:
                continue
            size = sum(len(q) for q in r.queries)
            if take and used + size > cap:
                break
            take.append(r)
            used += size
        for r in take:
            self.pending.remove(r)
        return take

    def _worker(self, ctx):
        while True:
            with self.lock:
                while not self.pending and not self.closed:
                    self.lock.wait()
                if not self.pending and self.closed:
                    return
                reqs = self._take()
                backlog = (self.batch and self.overlap_backlog is not None
                           and len(self.pending) >= self.overlap_backlog)
            try:
                if self.tunings:
                    ctx.set_tuning(**self.tunings.get(reqs[0].preset, self.base_tuning))
                arrays = batch_arrays(reqs)  # host work, beside the other worker's search
                search_batch(ctx, self.db, reqs, reqs[0].preset, self.index_chunks, arrays,
                             None if backlog else self.gpu_turn)
            except BaseException as e:  # surfaced by close()
                self.errors.append(e)
            t = self.now()
            with self.lock:
                for r in reqs:
                    r.done = t
                self.finished.extend(reqs)
                self.lock.notify_all()

    def warm(self, presets, queries):
        """Searches `queries` once per preset before serving (untimed): the
        contexts' scratch buffers grow to their working size and, with an
        index budget, each preset's seed index is built."""
        if self.tune_cache:
            letters, offsets = concat(list(queries))
            with self.gpu_turn:
                ctx = self.ctxs[0]
                batch = ResidentBatch(ctx, letters, offsets)
                try:
                    for preset in presets:
                        cfg = make_config(sensitivity=preset, index_chunks=self.index_chunks)
                        start = ctx.tuning()
                        self.tunings[preset] = ctx.autotune(self.db, batch, cfg, cache_path=self.tune_cache)[0]
                        ctx.set_tuning(**start)
                finally:
                    batch.close()
        for ctx in self.ctxs:
            for preset in presets:
                if self.tunings:
                    ctx.set_tuning(**self.tunings.get(preset, self.base_tuning))
                search_batch(ctx, self.db, [Request(-1, preset, list(queries))], preset, self.index_chunks,
                             gpu_turn=self.gpu_turn)

    def close(self):
        with self.lock:
            self.closed = True
            self.lock.notify_all()
        for t in self.threads:
            t.join()
        self.db.close()
        for c in self.ctxs:
            c.close()
        if self.errors:
            raise self.errors[0]


def poisson_stream(rng, n_requests, rate, max_queries, presets, q_mean=350, q_lo=20, q_hi=3000):
    """Requests of a serving stream: exponential gaps at `rate` per second,
    1..max_queries queries each (lengths lognormal), presets drawn uniformly."""
    from . import synth
    reqs, t = [], 0.0
    for k in range(n_requests):
        t += float(rng.exponential(1.0 / rate))
        nq = int(rng.integers(1, max_queries + 1))
        qs = [synth.random_protein(rng, L) for L in synth.lognormal_lengths(rng, nq, q_mean, q_lo, q_hi)]
        reqs.append((t, Request(k, str(rng.choice(presets)), qs)))
    return reqs


def run_stream(server: Server, stream):
    """Replays the stream in real time; returns the finished requests and the span."""
    start = time.perf_counter()
    for at, req in stream:
        delay = at - (time.perf_counter() - start)
        if delay > 0:
            time.sleep(delay)
        server.submit(req)
    with server.lock:
        while len(server.finished) < len(stream) and not server.errors:
            server.lock.wait(timeout=1.0)
    span = time.perf_counter() - start
    return list(server.finished), span


def latency_summary(finished, span):
    lat = sorted(r.done - r.arrival for r in finished)
    q = sum(len(r.queries) for r in finished)

    def pct(p):
        if not lat:
            return None
        k = min(len(lat) - 1, max(0, int(round(p / 100.0 * (len(lat) - 1)))))
        return lat[k]
    return {"requests": len(finished), "queries": q, "p50_s": pct(50), "p99_s": pct(99),
            "mean_s": statistics.fmean(lat) if lat else None, "queries_per_s": q / span if span > 0 else None,
            "mean_batch_requests": statistics.fmean(r.batch_size for r in finished) if finished else None}
