"""The tcgen05 building blocks (shared-memory descriptors of the canonical
K-major layout, kind::f16 MMA into tensor memory, commit to an mbarrier,
tcgen05.ld) against a CPU product of the same bf16-rounded operands."""
import ctypes

import numpy as np
import pytest

import gsn
from helpers import dev, empty, sync, torch

pytestmark = pytest.mark.gpu


def bf16(x):
    t = torch()
    return t.from_numpy(x).to(t.bfloat16).float().numpy()


@pytest.mark.parametrize("seed", [0, 1])
def test_tcgen05_gemm_matches_cpu_product(seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(128, 128)).astype(np.float32)
    b = rng.normal(size=(64, 128)).astype(np.float32)
    if seed == 1:  # structured operand: a banded Toeplitz filter like the SSIM passes
        w = np.exp(-0.5 * (np.arange(11) - 5) ** 2 / 1.5 ** 2)
        w /= w.sum()
        b = np.zeros((64, 128), np.float32)
        for n in range(64):
            for j in range(11):
                if 0 <= n + j < 128:
                    b[n, n + j] = w[j]
    t = torch()
    ad, bd = dev(a), dev(b)
    d = empty((128, 64), t.float32)
    fn = gsn.declare("gsn_tc_gemm_selftest", [ctypes.c_void_p] * 4)
    assert fn(ad.data_ptr(), bd.data_ptr(), d.data_ptr(), None) == 0
    sync()
    ref = bf16(a).astype(np.float64) @ bf16(b).astype(np.float64).T
    got = d.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.max(np.abs(ref)) + 1e-6
