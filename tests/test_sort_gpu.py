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
