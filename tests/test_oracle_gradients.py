"""CPU pinning of the oracle's backward: analytic FP64 gradients against FP64
central finite differences of the oracle's own forward model and loss, on the
scenes of the reference's solver tests (solver_test.cu), plus the reference's
known-answer Adam step."""
import numpy as np
import pytest

import oracle
import scenes
from solver_scenes import (active_fields, analytic, constant_target, differentiable_scene, finite_difference,
                           loss_of, overlapping_scene)


def close(a, fd, scale):
    return abs(a - fd) <= 2e-3 * abs(fd) + 1e-4 * scale


def test_loss_of_identical_images_is_zero():
    rng = np.random.default_rng(3)
    t = rng.integers(0, 256, (13, 17, 3), dtype=np.uint8)
    assert abs(oracle.loss(t / 255.0, t)) < 1e-12


def test_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    img = rng.uniform(0, 1, (19, 23, 3))
    t = rng.integers(0, 256, (19, 23, 3), dtype=np.uint8)
    g = oracle.loss_gradient(img, t)
    h = 1e-6
    for (y, x, c) in [(0, 0, 0), (9, 11, 1), (18, 22, 2), (5, 0, 2), (3, 17, 0)]:
        hi = img.copy()
        lo = img.copy()
        hi[y, x, c] += h
        lo[y, x, c] -= h
        fd = (oracle.loss(hi, t) - oracle.loss(lo, t)) / (2 * h)
        assert abs(g[y, x, c] - fd) < 1e-6 * max(1.0, abs(fd)) + 1e-9, (y, x, c, g[y, x, c], fd)


def test_loss_gradient_band_matches_full_image():
    rng = np.random.default_rng(6)
    img = rng.uniform(0, 1, (64, 40, 3))
    t = rng.integers(0, 256, (64, 40, 3), dtype=np.uint8)
    full = oracle.loss_gradient(img, t)
    band = oracle.loss_gradient(img, t, rows=(16, 32))
    assert np.array_equal(band[16:32], full[16:32])


@pytest.mark.parametrize("sh", [0, 1, 2, 3])
def test_single_gaussian_gradients_match_finite_differences(sh):
    # solver_test.cu:58-95 checks the sign of the update; the oracle is held to
    # the value of the derivative.
    params, cam, _ = differentiable_scene()
    target = constant_target(cam)
    bg = [0, 0, 0]
    a = analytic(params, cam, target, bg, sh)
    scale = np.abs(a["g58"]).max()
    for f in active_fields(sh):
        fd = finite_difference(params, cam, target, bg, sh, 0, f)
        assert abs(fd) > 1e-9
        assert close(a["g58"][f, 0], fd, scale), (f, a["g58"][f, 0], fd)
    inactive = [f for f in range(58) if f not in active_fields(sh)]
    assert np.all(a["g58"][inactive, 0] == 0)


@pytest.mark.parametrize("sh", [0, 3])
def test_overlapping_gaussians_with_background_match_finite_differences(sh):
    # solver_test.cu:97-154
    params, cam, bg = overlapping_scene()
    target = constant_target(cam)
    a = analytic(params, cam, target, bg, sh)
    scale = np.abs(a["g58"]).max()
    for i in range(3):
        for f in active_fields(sh):
            fd = finite_difference(params, cam, target, bg, sh, i, f)
            assert close(a["g58"][f, i], fd, scale), (i, f, a["g58"][f, i], fd)


def test_projection_statistic_matches_screen_translation_difference():
    # solver_test.cu:156-178: d loss / d(cx, cy) equals the summed d loss / d(u, v)
    params, cam, _ = differentiable_scene()
    target = constant_target(cam)
    a = analytic(params, cam, target, [0, 0, 0], 3)
    d = []
    for axis in range(2):
        hi = scenes.make_camera(9, 7)
        lo = scenes.make_camera(9, 7)
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
        d.append((loss_of(params, hi, target, [0, 0, 0], 3) - loss_of(params, lo, target, [0, 0, 0], 3)) / step)
    expected = np.hypot(d[0] * cam.width * 0.5, d[1] * cam.height * 0.5)
    assert abs(a["stats"][0, 0] - expected) < 2e-5 + expected * 0.002
    assert a["stats"][1, 0] == 1.0


def test_adam_step_after_history_reset_known_answer():
    # solver_test.cu:204-236: with zeroed moments at step 2 the opacity moves by
    # 0.025 * (0.1 / (1 - 0.9^2)) / sqrt(0.001 / (1 - 0.999^2)) against the gradient.
    n = 1
    p = np.zeros((58, n))
    m = np.zeros((58, n))
    v = np.zeros((58, n))
    g = np.zeros((58, n))
    g[9, 0] = -0.37
    oracle.adam(p, m, v, g, oracle.REFERENCE_LR, 2)
    factor = (0.1 / (1 - 0.9 ** 2)) / np.sqrt(0.001 / (1 - 0.999 ** 2))
    assert abs(p[9, 0] - 0.025 * factor) < 1e-12
    assert np.all(p[np.arange(58) != 9] == 0)


def test_absolute_statistics_exceed_signed_statistics():
    # solver_test.cu:309-356: the absolute sum dominates the signed one
    params = scenes.make_gaussians(1)
    params[0:3, 0] = [0, 0, 3]
    params[3:6, 0] = np.log(np.float32(0.5))
    params[10:58, 0] = 0
    cam = scenes.make_camera(9, 7)
    target = constant_target(cam)
    a = analytic(params, cam, target, [0, 0, 0], 0)
    assert a["abs_stats"][0] > a["stats"][0, 0] + 1e-5
