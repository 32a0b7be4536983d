"""GPU checks of the stable pair sort (gsn_sort_pairs) against numpy's stable
sort on the same keys: bit-exact keys and values, including ties, partial bit
ranges and empty / single-element inputs."""
import numpy as np
import pytest

import gsn
from helpers import dev, empty, sync, torch

pytestmark = pytest.mark.gpu


def run_sort(keys, values, begin_bit, end_bit):
    t = torch()
    n = len(keys)
    k, v = dev(keys.view(np.int32)), dev(values.view(np.int32))
    ka, va = empty((max(n, 1),), t.int32), empty((max(n, 1),), t.int32)
    ws_bytes = gsn.sort_pairs_workspace(n)
    ws = empty((max(ws_bytes, 1),), t.uint8)
    st, alt = gsn.sort_pairs(k.data_ptr(), v.data_ptr(), ka.data_ptr(), va.data_ptr(), n, begin_bit, end_bit,
                             ws.data_ptr(), ws_bytes)
    assert st == 0
    sync()
    rk, rv = (ka, va) if alt else (k, v)
    return rk.cpu().numpy()[:n].view(np.uint32), rv.cpu().numpy()[:n].view(np.uint32)


def expected(keys, values, begin_bit, end_bit):
    width = end_bit - begin_bit
    mask = np.uint64((1 << width) - 1)
    digit = (keys.astype(np.uint64) >> np.uint64(begin_bit)) & mask
    order = np.argsort(digit, kind="stable")
    return keys[order], values[order]


@pytest.mark.parametrize("n", [0, 1, 5, 4095, 4096, 4097, 100_000, 1_000_003])
@pytest.mark.parametrize("bits", [(0, 32), (0, 13), (4, 20)])
def test_sort_pairs_matches_stable_sort(n, bits):
    rng = np.random.default_rng(n + bits[1])
    keys = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    keys[: n // 3] = keys[n // 2: n // 2 + n // 3] if n > 6 else keys[: n // 3]  # force ties
    values = np.arange(n, dtype=np.uint32)
    k, v = run_sort(keys, values, *bits)
    ek, ev = expected(keys, values, *bits)
    assert np.array_equal(k, ek) and np.array_equal(v, ev)


def test_sort_pairs_rejects_bad_arguments():
    st, _ = gsn.sort_pairs(0, 0, 0, 0, 10, 0, 32, 0, 0)
    assert st != 0
    st, _ = gsn.sort_pairs(0, 0, 0, 0, 10, 0, 33, 0, 0)
    assert st != 0


@pytest.mark.parametrize("case", ["constant", "skewed_top_byte", "few_distinct"])
def test_sort_pairs_skewed_digits(case):
    """Digit distributions the histogram and the look-back must survive: one
    bucket holding every key, depth-like keys whose exponent byte barely varies,
    and a handful of distinct keys over 3M pairs (1,500 chunks of look-back)."""
    rng = np.random.default_rng(7)
    n = 3_000_000
    if case == "constant":
        keys = np.full(n, 0x40A00000, dtype=np.uint32)
    elif case == "skewed_top_byte":
        keys = rng.uniform(2.0, 30.0, n).astype(np.float32).view(np.uint32)
        keys[::97] = 0xFFFFFFFF  # culled entries sort last, as in the renderer
    else:
        keys = rng.integers(0, 5, n).astype(np.uint32) * 0x01010101
    values = np.arange(n, dtype=np.uint32)
    k, v = run_sort(keys, values, 0, 32)
    ek, ev = expected(keys, values, 0, 32)
    assert np.array_equal(k, ek) and np.array_equal(v, ev)


def test_sort_pairs_many_chunks_tile_bits():
    """8M records on 13 tile bits (two passes, 3,900 chunks per pass)."""
    rng = np.random.default_rng(11)
    n = 8_000_000
    keys = rng.integers(0, 6700, n).astype(np.uint32)
    values = rng.integers(0, 2 ** 31, n).astype(np.uint32)
    k, v = run_sort(keys, values, 0, 13)
    ek, ev = expected(keys, values, 0, 13)
    assert np.array_equal(k, ek) and np.array_equal(v, ev)


def run_scan(values, gather=None, valid=None, in_place=False):
    t = torch()
    n = len(values)
    if in_place:
        inp = out = dev(np.concatenate([values, [0]]).astype(np.int32))
    else:
        inp, out = dev(values.astype(np.int32)), empty((n + 1,), t.int32)
    g = dev(gather.astype(np.int32)) if gather is not None else None
    vd = dev(np.array([valid], dtype=np.int32)) if valid is not None else None
    ws_bytes = gsn.exclusive_scan_workspace(n)
    ws = empty((max(ws_bytes, 1),), t.uint8)
    st = gsn.exclusive_scan(inp.data_ptr(), g.data_ptr() if g is not None else 0, out.data_ptr(), n,
                            vd.data_ptr() if vd is not None else 0, ws.data_ptr(), ws_bytes)
    assert st == 0
    sync()
    return out.cpu().numpy()[:n + 1].astype(np.int64)


def expected_scan(values, gather=None, valid=None):
    entries = values[gather] if gather is not None else values.copy()
    if valid is not None:
        entries[valid:] = 0
    return np.concatenate([[0], np.cumsum(entries.astype(np.int64))])


@pytest.mark.parametrize("n", [1, 2047, 2048, 2049, 100_000, 1_200_000, 5_000_001])
def test_exclusive_scan_matches_cumulative_sum(n):
    """The one-pass scan (decoupled look-back over 2,048-entry chunks) against
    numpy's cumulative sum: plain, gathered through a permutation with a device
    valid count (the renderer's record scan in depth order), and in place (the
    density controller's use)."""
    rng = np.random.default_rng(n)
    values = rng.integers(0, 40, n).astype(np.int32)
    assert np.array_equal(run_scan(values), expected_scan(values))
    perm = rng.permutation(n).astype(np.int64)
    valid = int(n * 0.6)
    assert np.array_equal(run_scan(values, perm, valid), expected_scan(values, perm, valid))
    assert np.array_equal(run_scan(values, in_place=True), expected_scan(values))


def test_exclusive_scan_edge_cases():
    t = torch()
    out = dev(np.array([7], dtype=np.int32))
    ws = empty((gsn.exclusive_scan_workspace(0) or 1,), t.uint8)
    assert gsn.exclusive_scan(0, 0, out.data_ptr(), 0, 0, ws.data_ptr(), 16) == 0
    sync()
    assert out.cpu().numpy()[0] == 0
    values = np.zeros(3000, dtype=np.int32)
    assert np.array_equal(run_scan(values, valid=0), np.zeros(3001))
    # a workspace smaller than the count needs is rejected without launching
    buf = dev(np.ones(5000, dtype=np.int32))
    assert gsn.exclusive_scan(buf.data_ptr(), 0, buf.data_ptr(), 4999, 0, ws.data_ptr(), 16) != 0
