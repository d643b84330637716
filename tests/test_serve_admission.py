"""Admission of the continuous-batching server (drgpu/serve.py, CPU only).

A free worker takes the oldest queued request and, behind it, queued requests
of the same preset while the batch stays within max(merge_floor, merge_ratio x
the oldest request's letters) and the letter budget; requests of other presets
keep their place, and a request that does not fit stops the scan so that no
later request of that preset overtakes it.  The plain server takes one
request at a time.
"""
import types

import numpy as np

from drgpu import serve


def _req(rid, preset, letters):
    return serve.Request(rid, preset, [np.zeros(letters, np.uint8)])


def _server(pending, batch=True, budget=1_000_000, merge_ratio=1.0, merge_floor=64_000):
    return types.SimpleNamespace(pending=list(pending), batch=batch, budget=budget, merge_ratio=merge_ratio,
                                 merge_floor=merge_floor)


def _take(srv):
    return [r.rid for r in serve.Server._take(srv)]


def test_small_requests_share_a_batch_up_to_the_floor():
    srv = _server([_req(0, "fast", 10_000), _req(1, "fast", 20_000), _req(2, "sensitive", 5_000),
                   _req(3, "fast", 30_000), _req(4, "fast", 10_000)])
    assert _take(srv) == [0, 1, 3]  # 60,000 letters; request 4 would pass 64,000
    assert [r.rid for r in srv.pending] == [2, 4]


def test_a_large_request_runs_alone():
    srv = _server([_req(0, "default", 700_000), _req(1, "default", 1_000), _req(2, "default", 2_000)])
    assert _take(srv) == [0]  # the cap is its own size: nothing behind it delays it
    assert _take(srv) == [1, 2]


def test_a_request_that_does_not_fit_is_not_overtaken():
    srv = _server([_req(0, "fast", 40_000), _req(1, "fast", 50_000), _req(2, "fast", 1_000)])
    assert _take(srv) == [0]  # 1 does not fit beside 0, and 2 may not pass it
    assert _take(srv) == [1, 2]


def test_plain_budget_and_plain_server():
    srv = _server([_req(0, "fast", 700_000), _req(1, "fast", 200_000), _req(2, "fast", 200_000)], merge_ratio=None)
    assert _take(srv) == [0, 1]  # the 1M-letter budget alone
    srv = _server([_req(0, "fast", 10), _req(1, "fast", 10)], batch=False)
    assert _take(srv) == [0]
    assert _take(srv) == [1]
