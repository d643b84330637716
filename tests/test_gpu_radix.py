"""The device radix sort (drg_radix_sort) against numpy's stable sort.

It sorts the seed keys (seed::build, seed.rs:102), the hits (search.rs:178)
and the score pass's band and task keys.  LSD passes are only correct if each
pass is stable, so values are the input positions and must come out in the
order a stable sort gives.  Sizes cover empty input, one key, the 128-bit
load tail, tile edges (4,096 u32 / 3,072 u64 keys per tile) and many tiles;
bit ranges cover partial digits and bits above the range that must be
ignored.  The count is also handed over in device memory, with buffers sized
for a larger capacity.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def expect(keys, begin, end):
    mask = np.uint64((1 << (end - begin)) - 1) if end - begin < 64 else np.uint64((1 << 64) - 1)
    sub = (keys.astype(np.uint64) >> np.uint64(begin)) & mask
    order = np.argsort(sub, kind="stable")
    return keys[order], order.astype(np.uint32)


@pytest.mark.parametrize("dtype", [np.uint32, np.uint64])
@pytest.mark.parametrize("n", [0, 1, 3, 4095, 4096, 4097, 3071, 3072, 3073, 100003, 1 << 20])
def test_sort_pairs_full_range(ctx, dtype, n):
    r = np.random.Generator(np.random.PCG64(n + 17))
    bits = 8 * np.dtype(dtype).itemsize
    keys = r.integers(0, 1 << 62, n, dtype=np.uint64).astype(dtype) if bits == 64 else \
        r.integers(0, 1 << 32, n, dtype=np.uint64).astype(dtype)
    if n > 10:
        keys[::7] = keys[3]  # runs of equal keys: stability shows in the values
    vals = np.arange(n, dtype=np.uint32)
    gk, gv = ctx.radix_sort(keys, vals, 0, bits)
    ek, ev = expect(keys, 0, bits)
    assert np.array_equal(gk, ek)
    assert np.array_equal(gv, ev)


@pytest.mark.parametrize("dtype,begin,end", [(np.uint32, 0, 28), (np.uint32, 0, 23), (np.uint32, 13, 32),
                                             (np.uint64, 0, 45), (np.uint64, 13, 64), (np.uint64, 0, 27),
                                             (np.uint64, 5, 6)])
@pytest.mark.parametrize("on_device", [False, True])
def test_sort_bit_ranges(ctx, dtype, begin, end, on_device):
    r = np.random.Generator(np.random.PCG64(begin * 100 + end))
    n = 250001
    keys = r.integers(0, 1 << 63, n, dtype=np.uint64)
    if dtype == np.uint32:
        keys = keys.astype(np.uint32)
    keys[::11] = np.iinfo(dtype).max  # "no seed" keys: every bit set
    vals = np.arange(n, dtype=np.uint32)
    gk, gv = ctx.radix_sort(keys, vals, begin, end, count_on_device=on_device)
    _, ev = expect(keys, begin, end)
    assert np.array_equal(gv, ev)
    assert np.array_equal(gk, keys[ev])


@pytest.mark.parametrize("on_device", [False, True])
def test_sort_keys_only_skewed(ctx, on_device):
    # few distinct digits per pass (one tile-digit group holds most keys)
    r = np.random.Generator(np.random.PCG64(3))
    n = 700000
    keys = (r.integers(0, 4, n, dtype=np.uint64) << np.uint64(20)) | r.integers(0, 3, n, dtype=np.uint64)
    gk, _ = ctx.radix_sort(keys, None, 0, 40, count_on_device=on_device)
    assert np.array_equal(gk, np.sort(keys, kind="stable"))


def test_sort_sequence_shares_scratch(ctx):
    # Sorts of different pass counts and growing sizes one after another on
    # one context: they share the look-back area (its words carry the pass's
    # epoch), which must never hold another sort's histograms or stale words
    # of a reallocated block.
    r = np.random.Generator(np.random.PCG64(99))
    plan = [(np.uint64, 0, 64, 300000), (np.uint32, 0, 8, 5000), (np.uint64, 0, 16, 2000000),
            (np.uint32, 0, 32, 70000), (np.uint64, 20, 30, 4000000), (np.uint32, 3, 11, 9000),
            (np.uint64, 0, 64, 1 << 20), (np.uint32, 0, 24, 6000000), (np.uint64, 0, 8, 100)]
    for rep in range(3):
        for dtype, begin, end, n in plan:
            hi = 1 << 63 if dtype == np.uint64 else 1 << 32
            keys = r.integers(0, hi, n, dtype=np.uint64).astype(dtype)
            keys[::5] = keys[1]
            vals = np.arange(n, dtype=np.uint32)
            gk, gv = ctx.radix_sort(keys, vals, begin, end, count_on_device=bool(rep & 1))
            _, ev = expect(keys, begin, end)
            assert np.array_equal(gv, ev), (rep, dtype, begin, end, n)
            assert np.array_equal(gk, keys[ev])
