"""GPU tests of density control: the reference's density tests
(density_test.cu) through the C ABI, bit-exact comparison with the
reference's own DensityController on a large random case (same Philox
samples), the FP64/float oracle on the GPU's samples, and the Gaussian cap."""
import ctypes
import math

import numpy as np
import pytest

import gsn
import oracle
import scenes
from helpers import dev, host, sync, torch

pytestmark = pytest.mark.gpu

V, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float


def upload_params(params):
    """Copies a (58, n) float32 block into a raw cudaMalloc buffer (the controller
    takes ownership of blocks handed to it)."""
    n = params.shape[1]
    if n == 0:
        return 0
    p = gsn.device_alloc(params.nbytes)
    arr = np.ascontiguousarray(params, dtype=np.float32)
    gsn.memcpy(p, arr.ctypes.data, arr.nbytes)
    return p


def download_params(ptr, n):
    if n == 0 or not ptr:
        return np.zeros((58, 0), np.float32)
    return host(ptr, np.float32, 58 * n).reshape(58, n)


class Result:
    """DensityResult of density_test.cu:8-53: applies ControlDensity to a copy."""

    def __init__(self):
        self.ptr, self.count, self.changes = 0, 0, [0, 0]

    def apply(self, ctl, params_ptr, count, threshold=0.15, max_screen=0.0, abs_thr=0.0):
        p = 0
        if count > 0:
            p = gsn.device_alloc(58 * 4 * count)
            gsn.memcpy(p, params_ptr, 58 * 4 * count)
        st, newp, n, ch = ctl.control(p, count, 1.0, threshold, 0.01, 0.005, max_screen, 42, abs_thr)
        if self.ptr:
            gsn.device_free(self.ptr)
        self.ptr, self.count, self.changes = newp, n, ch
        self.parents = ctl.buffers()[0]
        return st == 0

    def params(self):
        return download_params(self.ptr, self.count)


def stats(values):
    return dev(np.asarray(values, dtype=np.float32))


def test_preserves_parameters_and_removes_low_opacity():
    g = scenes.make_gaussians(3)
    g[9, 1] = math.log(0.001 / 0.999)
    src = upload_params(g)
    ctl = gsn.Density()
    assert ctl.initialize(3, 3) == 0
    r = Result()
    assert r.apply(ctl, src, 3)
    assert r.count == 2
    assert list(host(r.parents, np.int32, 2)) == [0, 2]
    assert r.changes == [0, 1]
    out = r.params()
    assert np.array_equal(out[:, 0], g[:, 0]) and np.array_equal(out[:, 1], g[:, 2])


def test_clones_visible_gradient_and_clears_accumulated_statistics():
    g = scenes.make_gaussians(3)
    g[3:6] = np.log(np.float32(0.005))
    src = upload_params(g)
    ctl = gsn.Density()
    assert ctl.initialize(3, 3) == 0
    grads = stats([0.12, 0.16, 50, 50, 0, 0])
    radii = stats([1, 0, 1])
    ids = dev(np.array([0, 0, 1], dtype=np.int32))
    assert ctl.accumulate_observations(grads.data_ptr(), radii.data_ptr(), ids.data_ptr(), 3) == 0
    first = Result()
    assert first.apply(ctl, src, 3)
    assert first.count == 4
    assert list(host(first.parents, np.int32, 4)) == [0, 1, 2, -1]
    out = first.params()
    assert np.array_equal(out[:, 0], out[:, 3])
    second = Result()
    assert second.apply(ctl, first.ptr, first.count)
    assert second.count == 4 and second.changes[0] == 0


def test_splits_reproducibly_and_rescales_children():
    g = scenes.make_gaussians(1)
    g[3:6] = np.log(np.float32(0.2))
    src = upload_params(g)
    s = stats([1, 1])
    results = []
    ctls = []
    for _ in range(2):
        ctl = gsn.Density()
        assert ctl.initialize(1, 1) == 0
        assert ctl.accumulate(s.data_ptr(), s.data_ptr(), 1) == 0
        r = Result()
        assert r.apply(ctl, src, 1)
        results.append(r)
        ctls.append(ctl)
    a, b = results
    assert a.count == 2
    assert list(host(a.parents, np.int32, 2)) == [-1, -1]
    assert list(host(ctls[0].buffers()[2], np.int32, 2)) == [0, 0]
    pa, pb = a.params(), b.params()
    assert np.array_equal(pa, pb)
    for child in range(2):
        assert np.all(np.isfinite(pa[:, child]))
        assert np.all(np.abs(np.exp(pa[3:6, child].astype(np.float64)) - 0.125) < 1e-7)
        assert np.array_equal(pa[6:, child], g[6:, 0])
    assert np.abs(pa[0:3, 0] - pa[0:3, 1]).sum() > 1e-6


@pytest.mark.parametrize("threshold", [0.19, 0.21])
def test_averages_round_statistics_before_selecting(threshold):
    g = scenes.make_gaussians(1)
    g[3:6] = np.log(np.float32(0.005))
    src = upload_params(g)
    first, second = stats([0.1, 1]), stats([0.3, 1])
    ctl = gsn.Density()
    assert ctl.initialize(1, 1) == 0
    assert ctl.accumulate(first.data_ptr(), first.data_ptr(), 1) == 0
    assert ctl.accumulate(second.data_ptr(), second.data_ptr(), 1) == 0
    r = Result()
    assert r.apply(ctl, src, 1, threshold)
    assert r.count == (2 if threshold < 0.2 else 1)
    assert r.changes == [1 if threshold < 0.2 else 0, 0]


def test_prunes_oversized_gaussians_when_enabled():
    g = scenes.make_gaussians(2)
    g[3:6, 0] = np.log(np.float32(0.2))
    g[3:6, 1] = np.log(np.float32(0.01))
    src = upload_params(g)
    ctl = gsn.Density()
    assert ctl.initialize(2, 2) == 0
    r = Result()
    assert r.apply(ctl, src, 2, 0.15, 20)
    assert r.count == 1
    assert list(host(r.parents, np.int32, 1)) == [1]


@pytest.mark.parametrize("max_opacity", [0.8, 0.01])
def test_resets_opacity_without_changing_other_fields(max_opacity):
    g = scenes.make_gaussians(4)
    g[9] = [math.log(0.95 / 0.05), math.log(0.2 / 0.8), math.log(0.8 / 0.2), -9]
    src = upload_params(g)
    ctl = gsn.Density()
    assert ctl.initialize(4, 4) == 0
    assert ctl.reset_opacity(src, 4, max_opacity) == 0
    sync()
    out = download_params(src, 4)
    limit = np.float32(math.log(np.float32(max_opacity) / (np.float32(1.0) - np.float32(max_opacity))))
    expected = g.copy()
    expected[9] = np.minimum(g[9], limit)
    assert np.allclose(out, expected, rtol=0, atol=1e-6)
    assert np.array_equal(out[np.arange(58) != 9], g[np.arange(58) != 9])


def test_supports_all_pruned_and_empty_input():
    g = scenes.make_gaussians(2)
    g[9] = -12
    src = upload_params(g)
    ctl = gsn.Density()
    assert ctl.initialize(2, 2) == 0
    r = Result()
    assert r.apply(ctl, src, 2)
    assert r.count == 0 and r.ptr == 0
    empty = Result()
    assert empty.apply(ctl, 0, 0)
    assert empty.count == 0


def test_uses_signed_gradients_for_clones_and_absolute_gradients_for_splits():
    g = scenes.make_gaussians(6)
    for i in range(6):
        g[3:6, i] = np.log(np.float32(0.005 if i < 2 else 0.02))
    g[3:6, 5] = np.log(np.float32(0.01))
    src = upload_params(g)
    s = stats([0.0003, 0.0001, 0.0003, 0.0001, 0.0003, 0.0003, 1, 1, 1, 1, 1, 1])
    a = stats([0.001, 0.001, 0.0007, 0.001, 0.001, 0.0007])
    ctl = gsn.Density()
    assert ctl.initialize(6, 6) == 0
    assert ctl.accumulate(s.data_ptr(), a.data_ptr(), 6) == 0
    r = Result()
    assert r.apply(ctl, src, 6, 0.0002, 0.0, 0.0008)
    assert r.count == 10
    assert list(host(ctl.buffers()[2], np.int32, 10)) == [0, 1, 2, 5, 0, 5, 3, 4, 3, 4]
    assert list(host(r.parents, np.int32, 10)) == [0, 1, 2, 5, -1, -1, -1, -1, -1, -1]
    nxt = Result()
    assert nxt.apply(ctl, r.ptr, 10, 0.0002, 0.0, 0.0008)
    assert nxt.count == 10 and nxt.changes[0] == 0


@pytest.mark.parametrize("threshold", [0.00084, 0.00086])
def test_averages_absolute_statistics_with_shared_observation_counts(threshold):
    g = scenes.make_gaussians(1)
    g[3:6] = np.log(np.float32(0.02))
    src = upload_params(g)
    s = stats([0.0, 1.0])
    first, second = stats([0.0007]), stats([0.001])
    ctl = gsn.Density()
    assert ctl.initialize(1, 1) == 0
    assert ctl.accumulate(s.data_ptr(), first.data_ptr(), 1) == 0
    assert ctl.accumulate(s.data_ptr(), second.data_ptr(), 1) == 0
    r = Result()
    assert r.apply(ctl, src, 1, 0.0002, 0.0, threshold)
    assert r.count == (2 if threshold < 0.00085 else 1)


# ---------------------------------------------------------------- large cases
def random_case(n, seed):
    rng = np.random.default_rng(seed)
    params = scenes.random_gaussians(n, seed)
    params[3:6] = rng.normal(-4.0, 1.0, (3, n))
    params[9] = rng.normal(-1.0, 2.5, n)
    s = np.zeros(2 * n, dtype=np.float32)
    s[:n] = rng.exponential(3e-4, n)
    s[n:] = rng.integers(0, 2, n)
    a = (s[:n] * rng.uniform(1.0, 4.0, n)).astype(np.float32)
    return params, s, a


def run_gsn(params, s, a, rounds=2, extent=3.0, abs_thr=0.0008, max_screen=20.0, seed=7, cap=0):
    n = params.shape[1]
    ctl = gsn.Density()
    assert ctl.initialize(n, n) == 0
    if cap:
        ctl.set_max_gaussians(cap)
    sd, ad = dev(s), dev(a)
    for _ in range(rounds):
        assert ctl.accumulate(sd.data_ptr(), ad.data_ptr(), n) == 0
    src = upload_params(params)
    st, p, m, ch = ctl.control(src, n, extent, 0.0002, 0.01, 0.005, max_screen, seed, abs_thr)
    assert st == 0
    sync()
    samples_ptr, _, _, _ = ctl.internals()
    hist, control, parents = ctl.buffers()
    out = dict(params=download_params(p, m), count=m, changes=ch, parents=host(parents, np.int32, m),
               history=host(hist, np.int32, m), samples_ptr=samples_ptr, ctl=ctl)
    gsn.device_free(p) if p else None
    return out


def run_ref(params, s, a, rounds=2, extent=3.0, abs_thr=0.0008, max_screen=20.0, seed=7):
    n = params.shape[1]
    h = V()
    oracle.ref_fn("ref_density_create", [ctypes.POINTER(V)])(ctypes.byref(h))
    assert oracle.ref_fn("ref_density_initialize", [V, I, I])(h, n, n) == 0
    sd, ad = dev(s), dev(a)
    acc = oracle.ref_fn("ref_density_accumulate", [V, V, V, I])
    for _ in range(rounds):
        assert acc(h, V(sd.data_ptr()), V(ad.data_ptr()), n) == 0
    src = V(upload_params(params))
    cnt = I(n)
    ch = (I * 2)()
    ctrl = oracle.ref_fn("ref_density_control", [V, ctypes.POINTER(V), ctypes.POINTER(I), F, F, F, F, F,
                                                 ctypes.c_ulonglong, V, F])
    assert ctrl(h, ctypes.byref(src), ctypes.byref(cnt), extent, 0.0002, 0.01, 0.005, max_screen, seed,
                ctypes.cast(ch, V), abs_thr) == 0
    m = cnt.value
    hp, cp, pp = V(), V(), V()
    oracle.ref_fn("ref_density_get", [V, ctypes.POINTER(V), ctypes.POINTER(V), ctypes.POINTER(V)])(
        h, ctypes.byref(hp), ctypes.byref(cp), ctypes.byref(pp))
    out = dict(params=download_params(src.value, m), count=m, changes=[ch[0], ch[1]],
               parents=host(pp.value, np.int32, m), history=host(hp.value, np.int32, m))
    if src.value:
        gsn.device_free(src.value)
    oracle.ref_fn("ref_density_destroy", [V])(h)
    return out


def test_large_random_case_bit_exact_against_reference():
    if not oracle.ref_available():
        pytest.skip("reference CUDA build not available")
    params, s, a = random_case(60_000, 3)
    mine = run_gsn(params, s, a)
    ref = run_ref(params, s, a)
    assert mine["count"] == ref["count"] and mine["changes"] == ref["changes"]
    assert mine["count"] != params.shape[1]
    assert np.array_equal(mine["parents"], ref["parents"])
    assert np.array_equal(mine["history"], ref["history"])
    assert np.array_equal(mine["params"].view(np.uint32), ref["params"].view(np.uint32))


def test_large_random_case_matches_oracle():
    params, s, a = random_case(20_000, 5)
    mine = run_gsn(params, s, a, rounds=1)
    n = params.shape[1]
    counts4 = oracle.density_counts(params, s[:n], a, s[n:].astype(np.uint32), 0.0002, 0.03, 0.005, 0.3, 1, 0.0008)
    z = int(counts4[:, 2].sum())
    samples = host(mine["samples_ptr"], np.float32, max(6 * z, 1))
    out, parents, hist = oracle.density_apply(params, counts4, samples)
    assert out.shape[1] == mine["count"]
    assert np.array_equal(parents, mine["parents"])
    assert np.array_equal(hist, mine["history"])
    assert np.allclose(out, mine["params"], rtol=2e-6, atol=2e-6)
    # the samples are standard normal
    assert abs(samples[: 6 * z].mean()) < 0.05 and abs(samples[: 6 * z].std() - 1) < 0.05


def test_cap_limits_growth_in_id_order():
    params, s, a = random_case(20_000, 9)
    free = run_gsn(params, s, a)
    assert free["count"] > 20_000
    cap = 20_000 + (free["count"] - 20_000) // 2
    capped = run_gsn(params, s, a, cap=cap)
    assert capped["count"] <= cap
    assert capped["count"] >= cap - 1
    # survivors and the accepted additions are a prefix (in id order) of the free run's decisions
    assert np.all(np.diff(capped["parents"][: np.sum(capped["history"] >= 0)]) > 0)
