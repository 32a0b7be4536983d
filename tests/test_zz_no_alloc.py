"""GPU test of gsn_sort_pairs_noalloc, the allocation-free variant of the pair sort.

It exists for callers that cannot allocate device memory (for example code under
an allocator that owns the whole device budget, or loops that cannot take the
synchronisation cudaMalloc implies); its scratch is a static device array of the
library. Each call must give exactly what gsn_sort_pairs gives with a
caller-provided workspace, including on a second call that reuses the scratch
left behind by the first, and counts above the stated maximum must be refused
without launching anything.

The file name makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

import gsn
from helpers import dev, empty, sync, torch

pytestmark = pytest.mark.gpu

MAX_COUNT = 16777216  # GSN_SORT_NOALLOC_MAX_COUNT in include/gsn.h


def noalloc():
    return gsn.declare("gsn_sort_pairs_noalloc",
                       [ctypes.c_void_p] * 4 + [ctypes.c_int] * 3 + [ctypes.POINTER(ctypes.c_int), ctypes.c_void_p])


def sort_both(keys, values, begin_bit, end_bit):
    """(result of gsn_sort_pairs, result of gsn_sort_pairs_noalloc) on copies of the same input."""
    t = torch()
    n = len(keys)
    outs = []
    for variant in ("workspace", "noalloc"):
        k, v = dev(keys.view(np.int32)), dev(values.view(np.int32))
        ka, va = empty((n,), t.int32), empty((n,), t.int32)
        if variant == "workspace":
            ws_bytes = gsn.sort_pairs_workspace(n)
            ws = empty((ws_bytes,), t.uint8)
            st, alt = gsn.sort_pairs(k.data_ptr(), v.data_ptr(), ka.data_ptr(), va.data_ptr(), n, begin_bit,
                                     end_bit, ws.data_ptr(), ws_bytes)
        else:
            a = ctypes.c_int()
            st = noalloc()(k.data_ptr(), v.data_ptr(), ka.data_ptr(), va.data_ptr(), n, begin_bit, end_bit,
                           ctypes.byref(a), None)
            alt = a.value
        assert st == 0, (variant, st)
        sync()
        rk, rv = (ka, va) if alt else (k, v)
        outs.append((rk.cpu().numpy().view(np.uint32), rv.cpu().numpy().view(np.uint32)))
    return outs


def test_noalloc_sort_matches_workspace_sort_on_two_calls_in_a_row():
    rng = np.random.default_rng(42)
    # first call: a large full-width sort; second call: a smaller one on fewer
    # bits, which reuses (a prefix of) the scratch the first call left behind
    for n, bits in ((1_000_003, (0, 32)), (70_001, (0, 13))):
        keys = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 4] = keys[n // 2: n // 2 + n // 4]  # ties
        values = rng.permutation(n).astype(np.uint32)
        (k0, v0), (k1, v1) = sort_both(keys, values, *bits)
        assert np.array_equal(k0, k1)
        assert np.array_equal(v0, v1)
        digits = (keys.astype(np.uint64) >> np.uint64(bits[0])) & np.uint64((1 << (bits[1] - bits[0])) - 1)
        order = np.argsort(digits, kind="stable")
        assert np.array_equal(v1, values[order])


def test_noalloc_sort_refuses_counts_above_its_maximum():
    a = ctypes.c_int(-1)
    # null pointers: the size check must refuse before anything is touched
    st = noalloc()(None, None, None, None, MAX_COUNT + 1, 0, 32, ctypes.byref(a), None)
    assert st == -4  # GSN_ERR_CAPACITY
    assert a.value == 0
