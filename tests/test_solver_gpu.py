"""GPU parity of the backward path: loss gradient, screen-space backward, chain
rule and Adam against the reference's own CUDA kernels and the FP64 oracle,
plus the reference's solver tests (solver_test.cu) run through the C ABI."""
import ctypes
import math

import numpy as np
import pytest

import gsn
import oracle
import scenes
from helpers import RefRenderer, dev, empty, host, sync, torch
from solver_scenes import (active_fields, analytic, constant_target, differentiable_scene, finite_difference,
                           loss_of, overlapping_scene)

pytestmark = pytest.mark.gpu

V, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float


def need_ref():
    if not oracle.ref_available():
        pytest.skip("reference CUDA build (oracle/_ref) not available")


def seeded_target(cam, seed=1, sh=3):
    """Target of the single-step case: a second 4,096-Gaussian set (seed 1)."""
    p = scenes.random_gaussians(4096, seed)
    img = oracle.render_params(p, cam, [1, 1, 1], sh)
    return np.clip(np.rint(img * 255.0), 0, 255).astype(np.uint8)


class Frame:
    """One rendered frame of gs-native plus the solver's stage outputs."""

    def __init__(self, params, cam, target, bg, sh, lr=1e-4):
        t = torch()
        self.n = params.shape[1]
        self.cam, self.sh, self.bg = cam, sh, bg
        self.p = dev(params)
        self.target = dev(target)
        self.image = empty((cam.height, cam.width, 3), t.float32)
        self.renderer = gsn.Renderer()
        self.solver = gsn.Solver()
        assert self.renderer.render(self.p.data_ptr(), self.n, cam, bg, self.image.data_ptr(), sh) == 0

    def image_gradients(self):
        ptr = self.solver.image_gradients(self.cam, self.image.data_ptr(), self.target.data_ptr())
        sync()
        return ptr

    def screen(self):
        self.image_gradients()
        ptr = self.solver.screen_gradients(self.cam, self.renderer, self.image.data_ptr(), self.p.data_ptr(), self.n)
        sync()
        return host(ptr, np.float32, 12 * self.n).reshape(self.n, 12)


def ref_image_gradients(image, target, cam):
    t = torch()
    g = empty((cam.height, cam.width, 3), t.float32)
    fn = oracle.ref_fn("ref_image_gradients", [V, V, V, I, I])
    assert fn(V(image.data_ptr()), V(target.data_ptr()), V(g.data_ptr()), cam.width, cam.height) == 0
    return g.cpu().numpy()


def ref_screen_gradients(frame, image_grad_ptr):
    t = torch()
    n = frame.n
    b = frame.renderer.buffers()
    grads = empty((58, n), t.float32)
    absolute = empty((2, n), t.float32)
    fn = oracle.ref_fn("ref_splat_gradients", [V] * 7 + [V, V, V, I])
    assert fn(V(b.tile_gaussian_ids), V(b.tile_offsets), V(b.means), V(b.conic_opacity), V(b.colors),
              V(frame.image.data_ptr()), V(image_grad_ptr), ctypes.byref(frame.cam), V(grads.data_ptr()),
              V(absolute.data_ptr()), n) == 0
    return grads.cpu().numpy(), absolute.cpu().numpy()


def rows_close(mine, ref, rel=1e-4, floor=1e-5):
    """Per row: |a - b| <= rel * |b| + floor * max|b| (float-atomic summation order)."""
    scale = np.abs(ref).max(axis=-1, keepdims=True)
    bad = np.abs(mine - ref) > rel * np.abs(ref) + floor * scale
    return not bad.any(), np.argwhere(bad)[:5]


def single_step(sh=3):
    params, cam = scenes.single_step_scene()
    target = seeded_target(cam)
    return params, cam, target


def test_image_gradients_match_reference_and_oracle():
    params, cam, target = single_step()
    f = Frame(params, cam, target, [1, 1, 1], 3)
    mine = host(f.image_gradients(), np.float32, cam.pixels * 3).reshape(cam.height, cam.width, 3)
    img = f.image.cpu().numpy().astype(np.float64)
    expected = oracle.loss_gradient(img, target)
    scale = np.abs(expected).max()
    assert np.abs(mine - expected).max() < 1e-4 * scale
    if oracle.ref_available():
        ref = ref_image_gradients(f.image, f.target, cam)
        # same filter tap order as the reference: equal to float rounding
        assert np.abs(mine - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.parametrize("size", [(9, 7), (33, 65), (128, 128), (101, 77)])
def test_loss_value_fp64_matches_oracle(size):
    rng = np.random.default_rng(size[0])
    cam = scenes.make_camera(*size)
    img = rng.uniform(0, 1, (size[1], size[0], 3)).astype(np.float32)
    target = rng.integers(0, 256, (size[1], size[0], 3), dtype=np.uint8)
    s = gsn.Solver()
    s.set_compute_loss(True)
    ti, tt = dev(img), dev(target)
    s.image_gradients(cam, ti.data_ptr(), tt.data_ptr())
    loss, l1, ssim, psnr = s.loss()
    expected = oracle.loss(img.astype(np.float64), target)
    assert abs(loss - expected) < 1e-6
    mse = np.mean((img.astype(np.float64) - target / 255.0) ** 2)
    assert abs(psnr - (-10 * math.log10(mse))) < 1e-4


def test_screen_gradients_match_reference_kernel():
    need_ref()
    params, cam, target = single_step()
    f = Frame(params, cam, target, [1, 1, 1], 3)
    mine = f.screen()
    gptr = f.solver.image_gradients(f.cam, f.image.data_ptr(), f.target.data_ptr())
    ref_rows, ref_abs = ref_screen_gradients(f, gptr)
    ok, where = rows_close(mine[:, :9].T, ref_rows[:9])
    assert ok, where
    ok, where = rows_close(mine[:, 9:11].T, ref_abs)
    assert ok, where
    assert np.count_nonzero(ref_rows[:9]) > 1000


@pytest.mark.parametrize("sh", [0, 3])
def test_screen_gradients_match_oracle_on_reference_scenes(sh):
    params, cam, bg = overlapping_scene()
    target = constant_target(cam)
    f = Frame(params, cam, target, bg, sh)
    mine = f.screen()
    a = analytic(params, cam, target, bg, sh)
    # FP32 against FP64: measured at most 2.6e-5 relative on these scenes
    ok, where = rows_close(mine[:, :9].T.astype(np.float64), a["g9"], rel=1e-4, floor=1e-6)
    assert ok, where


@pytest.mark.parametrize("sh", [0, 1, 2, 3])
def test_mapped_gradients_match_reference_kernel_to_rounding(sh):
    # Same screen-space input for both; the chain rule mirrors the reference's
    # expressions, so results agree to float rounding (the fused kernel's FMA
    # contraction may differ from the reference's stand-alone kernel).
    need_ref()
    params, cam, target = single_step()
    f = Frame(params, cam, target, [1, 1, 1], sh)
    screen = f.screen()
    t = torch()
    mine = empty((58, f.n), t.float32)
    f.solver.map_gradients(cam, f.renderer, f.p.data_ptr(), f.n, sh, mine.data_ptr())
    sync()
    ref = np.zeros((58, f.n), dtype=np.float32)
    ref[:9] = screen[:, :9].T
    rg = dev(ref)
    fn = oracle.ref_fn("ref_map_gradients", [V, V, V, I, I])
    assert fn(V(f.p.data_ptr()), ctypes.byref(cam), V(rg.data_ptr()), f.n, sh) == 0
    a, b = mine.cpu().numpy(), rg.cpu().numpy()
    ok, where = rows_close(a, b, rel=1e-4, floor=1e-6)
    assert ok, where
    assert np.mean(a == b) > 0.9


def test_mapped_gradients_match_oracle():
    params, cam, bg = overlapping_scene()
    target = constant_target(cam)
    for sh in range(4):
        f = Frame(params, cam, target, bg, sh)
        f.screen()
        t = torch()
        g = empty((58, f.n), t.float32)
        f.solver.map_gradients(cam, f.renderer, f.p.data_ptr(), f.n, sh, g.data_ptr())
        sync()
        a = analytic(params, cam, target, bg, sh)
        # FP32 against FP64: measured at most 3.8e-6 relative
        ok, where = rows_close(g.cpu().numpy().astype(np.float64), a["g58"], rel=1e-4, floor=1e-6)
        assert ok, (sh, where)


@pytest.mark.parametrize("sh", [0, 1, 2, 3])
def test_mapped_gradients_match_finite_differences(sh):
    """Magnitudes, not only signs: every active parameter gradient of the three
    overlapping Gaussians (coloured background) against FP64 central differences
    of the oracle's loss (h = 5e-4), within 1e-4 relative; derivatives below a
    thousandth of their row's largest get that as their scale. Measured at most
    5.1e-6."""
    params, cam, bg = overlapping_scene()
    target = constant_target(cam)
    f = Frame(params, cam, target, bg, sh)
    f.screen()
    t = torch()
    g = empty((58, f.n), t.float32)
    f.solver.map_gradients(cam, f.renderer, f.p.data_ptr(), f.n, sh, g.data_ptr())
    sync()
    g58 = g.cpu().numpy().astype(np.float64)
    a = analytic(params, cam, target, bg, sh)
    checked = 0
    for i in range(3):
        for field in active_fields(sh):
            d = finite_difference(params, cam, target, bg, sh, i, field)
            scale = max(abs(d), 1e-3 * np.abs(a["g58"][field]).max())
            assert abs(g58[field, i] - d) <= 1e-4 * scale, (i, field, g58[field, i], d)
            checked += 1
    assert checked == 3 * len(active_fields(sh))


def run_step(frame, lr=1e-4):
    assert frame.solver.iterate(frame.cam, frame.renderer, frame.image.data_ptr(), frame.target.data_ptr(),
                                frame.p.data_ptr(), frame.n, lr, frame.sh) == 0
    sync()


def test_iterate_matches_reference_solver():
    need_ref()
    params, cam, target = single_step()
    f = Frame(params, cam, target, [1, 1, 1], 3)
    run_step(f)
    mine = f.p.cpu().numpy()
    # reference Render + Solver::Iterate on a copy of the same inputs
    t = torch()
    rp = dev(params)
    rimg = empty((cam.height, cam.width, 3), t.float32)
    rr = RefRenderer()
    assert rr.render(rp.data_ptr(), f.n, cam, [1, 1, 1], rimg.data_ptr(), 3) == 0
    h = V()
    oracle.ref_fn("ref_solver_create", [ctypes.POINTER(V)])(ctypes.byref(h))
    it = oracle.ref_fn("ref_solver_iterate", [V, V, V, V, V, V, I, F, I])
    assert it(h, ctypes.byref(cam), rr.h, V(rimg.data_ptr()), V(f.target.data_ptr()), V(rp.data_ptr()), f.n,
              1e-4, 3) == 0
    ref = rp.cpu().numpy()
    oracle.ref_fn("ref_solver_destroy", [V])(h)
    # Adam's first step moves every parameter with a nonzero gradient by about
    # its learning rate, so differences are either tiny or sign flips of
    # gradients that are themselves at rounding level.
    diff = np.abs(mine - ref)
    moved = np.abs(ref - params)
    assert np.mean(diff <= 1e-6 + 1e-3 * moved) > 0.999
    assert np.isfinite(mine).all()


@pytest.mark.parametrize("n", [4099, 4096 + 66, 130, 61, 3])
def test_adam_matches_fp32_adam_of_mapped_gradients_on_ragged_counts(n):
    """Counts that are not multiples of the warp or CTA width (rows starting at
    every 16-byte phase, partial last blocks): the fused update must equal FP32
    Adam (solver.cu:651-689) applied to the kernel's own mapped gradients."""
    t = torch()
    _, cam = scenes.single_step_scene()
    params = scenes.random_gaussians(n, 5)
    target = seeded_target(cam)
    f = Frame(params, cam, target, [1, 1, 1], 3)
    f.screen()
    grads = empty((58, n), t.float32)
    f.solver.map_gradients(cam, f.renderer, f.p.data_ptr(), n, 3, grads.data_ptr())
    sync()
    g = grads.cpu().numpy()
    run_step(f, lr=1e-4)
    m_ptr, v_ptr, it = f.solver.moments()
    assert it == 1
    m = host(m_ptr, np.float32, 58 * n).reshape(58, n)
    v = host(v_ptr, np.float32, 58 * n).reshape(58, n)
    p = f.p.cpu().numpy()
    lr = np.empty((58, 1), np.float32)
    lr[0:3], lr[3:6], lr[6:9], lr[9] = 1e-4, 0.005, 0.001, 0.025
    lr[10:] = 0.0025 / 20
    lr[[10, 26, 42]] = 0.0025
    f32 = np.float32
    em = f32(0.1) * g
    ev = f32(0.001) * g * g
    c1, c2 = f32(1 / (1 - 0.9)), f32(1 / (1 - 0.999))
    ep = params - lr * (em * c1) / (np.sqrt(ev * c2) + f32(1e-15))
    # screen gradients are re-accumulated by the iterate (atomic order), so
    # compare to rounding; a misplaced row or tile would be off by O(1)
    assert np.mean(np.abs(m - em) <= 1e-3 * np.abs(em) + 1e-12) > 0.999
    assert np.mean(np.abs(v - ev) <= 2e-3 * np.abs(ev) + 1e-18) > 0.999
    assert np.mean(np.abs(p - ep) <= 1e-6 + 1e-3 * np.abs(ep - params)) > 0.999
    # rows with exactly zero gradient keep their value and zero moments
    zero = g == 0
    assert np.array_equal(p[zero], params[zero]) and not m[zero].any() and not v[zero].any()


@pytest.mark.parametrize("sh", [0, 1, 2, 3])
def test_update_directions_match_finite_differences(sh):
    # solver_test.cu:58-95
    params, cam, _ = differentiable_scene()
    target = constant_target(cam)
    f = Frame(params, cam, target, [0, 0, 0], sh)
    run_step(f)
    after = f.p.cpu().numpy()
    assert np.isfinite(after).all()
    verified = 0
    for field in range(58):
        if field not in active_fields(sh):
            assert after[field, 0] == params[field, 0]
            continue
        d = finite_difference(params, cam, target, [0, 0, 0], sh, 0, field)
        assert abs(d) > 1e-9
        assert d * (after[field, 0] - params[field, 0]) < 0, field
        verified += 1
    assert verified == 10 + 3 * (sh + 1) ** 2


@pytest.mark.parametrize("sh", [0, 3])
def test_overlapping_gaussians_with_background_match_finite_differences(sh):
    # solver_test.cu:97-154
    params, cam, bg = overlapping_scene()
    target = constant_target(cam)
    f = Frame(params, cam, target, bg, sh)
    run_step(f)
    after = f.p.cpu().numpy()
    for i in range(3):
        for field in active_fields(sh):
            d = finite_difference(params, cam, target, bg, sh, i, field)
            assert d * (after[field, i] - params[field, i]) < 0, (i, field)


def screen_translation_derivative(params, cam, target, sh):
    d = []
    for axis in range(2):
        hi = scenes.make_camera(cam.width, cam.height)
        lo = scenes.make_camera(cam.width, cam.height)
        for c in (hi, lo):
            for k in range(9):
                c.R_c_w[k] = cam.R_c_w[k]
        if axis == 0:
            hi.cx += 0.001
            lo.cx -= 0.001
            step = hi.cx - lo.cx
        else:
            hi.cy += 0.001
            lo.cy -= 0.001
            step = hi.cy - lo.cy
        d.append((loss_of(params, hi, target, [0, 0, 0], sh) - loss_of(params, lo, target, [0, 0, 0], sh)) / step)
    return np.hypot(d[0] * cam.width * 0.5, d[1] * cam.height * 0.5)


def test_projection_statistic_matches_screen_translation_difference():
    # solver_test.cu:156-178
    params, cam, _ = differentiable_scene()
    target = constant_target(cam)
    f = Frame(params, cam, target, [0, 0, 0], 3)
    run_step(f)
    sp, _ = f.solver.statistics()
    stats = host(sp, np.float32, 2)
    expected = screen_translation_derivative(params, cam, target, 3)
    assert abs(stats[0] - expected) < 2e-5 + expected * 0.002
    assert stats[1] == 1.0


def test_projection_gradient_matches_across_ssim_blocks_and_partial_edges():
    # solver_test.cu:276-307
    params, _, R = differentiable_scene()
    cam = scenes.make_camera(33, 65)
    scenes.set_pose(cam, R, np.zeros(3, np.float32))
    params[3:6, 0] = np.log(np.array([3.0, 2.5, 1.8], dtype=np.float32))
    y, x = np.mgrid[0:65, 0:33]
    target = np.stack([120 + (3 * x + y) % 100, 100 + (x + 2 * y) % 120, 140 + (2 * x + 3 * y) % 100],
                      axis=-1).astype(np.uint8)
    f = Frame(params, cam, target, [0, 0, 0], 3)
    run_step(f)
    sp, _ = f.solver.statistics()
    stats = host(sp, np.float32, 2)
    expected = screen_translation_derivative(params, cam, target, 3)
    assert expected > 1e-6
    assert abs(stats[0] - expected) < 2e-5 + expected * 0.002
    assert stats[1] == 1.0


def test_parent_permutation_preserves_subsequent_updates():
    # solver_test.cu:180-202
    params = scenes.make_gaussians(2)
    cam = scenes.make_camera(19, 17)
    target = np.full((17, 19, 3), 180, dtype=np.uint8)
    a = Frame(params, cam, target, [0, 0, 0], 1)
    b = Frame(params, cam, target, [0, 0, 0], 1)
    run_step(a)
    run_step(b)
    values = b.p.cpu().numpy()[:, ::-1].copy()
    b.p.copy_(torch().from_numpy(values))
    parents = dev(np.array([1, 0], dtype=np.int32))
    assert b.solver.remap(parents.data_ptr(), 2) == 0
    for fr in (a, b):
        fr.target.fill_(20)
        assert fr.renderer.render(fr.p.data_ptr(), 2, cam, [0, 0, 0], fr.image.data_ptr(), 1) == 0
        run_step(fr)
    pa, pb = a.p.cpu().numpy(), b.p.cpu().numpy()
    assert np.abs(pa[:, 0] - pb[:, 1]).max() < 2e-6
    assert np.abs(pa[:, 1] - pb[:, 0]).max() < 2e-6


ADAM_FACTOR = (0.1 / (1 - 0.9 ** 2)) / math.sqrt(0.001 / (1 - 0.999 ** 2))


def test_opacity_history_reset_uses_zero_moments_at_current_step():
    # solver_test.cu:204-220
    params, cam, _ = differentiable_scene()
    target = np.full((7, 9, 3), 200, dtype=np.uint8)
    f = Frame(params, cam, target, [0, 0, 0], 0)
    run_step(f)
    values = f.p.cpu().numpy()
    values[9, 0] = math.log(0.01 / 0.99)
    f.p.copy_(torch().from_numpy(values))
    assert f.solver.reset_opacity_history() == 0
    assert f.renderer.render(f.p.data_ptr(), 1, cam, [0, 0, 0], f.image.data_ptr(), 0) == 0
    run_step(f)
    actual = f.p.cpu().numpy()
    assert abs((actual[9, 0] - values[9, 0]) - 0.025 * ADAM_FACTOR) < 2e-6


def test_new_parent_starts_with_zero_history():
    # solver_test.cu:221-236
    params, cam, _ = differentiable_scene()
    target = np.full((7, 9, 3), 200, dtype=np.uint8)
    f = Frame(params, cam, target, [0, 0, 0], 0)
    run_step(f)
    before = f.p.cpu().numpy()
    parents = dev(np.array([-1], dtype=np.int32))
    assert f.solver.remap(parents.data_ptr(), 1) == 0
    assert f.renderer.render(f.p.data_ptr(), 1, cam, [0, 0, 0], f.image.data_ptr(), 0) == 0
    run_step(f)
    actual = f.p.cpu().numpy()
    assert abs((actual[9, 0] - before[9, 0]) - 0.025 * ADAM_FACTOR) < 2e-6


def test_gradients_cross_gaussian_batch_boundary():
    # solver_test.cu:237-274
    n = 257
    params = scenes.make_gaussians(n)
    i = np.arange(n, dtype=np.float32)
    params[0], params[1] = 0.1, -0.1
    params[2] = np.float32(3.0) + np.float32(0.001) * i
    params[3:6] = np.log(np.float32(0.8))
    params[9] = -4.4
    params[10] += np.float32(0.1) * np.sin(i)
    params = np.ascontiguousarray(params[:, ::-1])
    cam = scenes.make_camera(9, 7)
    target = constant_target(cam)
    f = Frame(params, cam, target, [0, 0, 0], 0)
    run_step(f)
    after = f.p.cpu().numpy()
    assert np.isfinite(after).all()
    for g in (0, 1, 128, 255, 256):
        for field in (9, 10, 26, 42):
            d = finite_difference(params, cam, target, [0, 0, 0], 0, g, field)
            assert abs(d) > 1e-9
            assert d * (after[field, g] - params[field, g]) < 0, (g, field)


def test_absolute_statistics_exceed_signed_statistics():
    # solver_test.cu:309-356 (magnitude against the FP64 oracle)
    params = scenes.make_gaussians(1)
    params[0:3, 0] = [0, 0, 3]
    params[3:6, 0] = np.log(np.float32(0.5))
    params[10:58, 0] = 0
    cam = scenes.make_camera(9, 7)
    target = constant_target(cam)
    f = Frame(params, cam, target, [0, 0, 0], 0)
    run_step(f)
    sp, ap = f.solver.statistics()
    stats, abs_stats = host(sp, np.float32, 2), host(ap, np.float32, 1)
    a = analytic(params, cam, target, [0, 0, 0], 0)
    expected = a["abs_stats"][0]
    assert expected > 1e-5
    assert abs(abs_stats[0] - expected) < 2e-5 + expected * 0.002
    assert abs_stats[0] > stats[0] + 1e-5
