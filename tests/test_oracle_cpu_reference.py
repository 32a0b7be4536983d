"""The reference's own CPU reference (test/cpu_reference.h RenderReference and
ComputeLoss), compiled unmodified against the OpenCV shim into
oracle/_ref/libgsref_cpu.so, checked on the CPU: its loss against OpenCV's
own filters (tests/golden/cv_loss_golden.npz, made with cv2 by
make_cv_loss_golden.py), and both against the FP64 oracle on the reference's
renderer test scenes and the seeded 4,096-Gaussian single-step scene."""
import os

import numpy as np
import pytest

import oracle
import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cv_loss_golden.npz")


def need_cpu_ref():
    if not oracle.ref_cpu_available():
        pytest.skip("oracle/_ref/libgsref_cpu.so not built (no reference tree where build() ran)")


def test_compute_loss_matches_opencv_golden():
    need_cpu_ref()
    g = np.load(GOLDEN)
    for i in range(int(g["cases"])):
        got = oracle.ref_cpu_loss(g[f"image{i}"], g[f"target{i}"])
        assert abs(got - float(g[f"loss{i}"])) < 1e-13, i


def test_compute_loss_matches_oracle_loss():
    need_cpu_ref()
    g = np.load(GOLDEN)
    for i in range(int(g["cases"])):
        image, target = g[f"image{i}"], g[f"target{i}"]
        assert abs(oracle.ref_cpu_loss(image, target) - oracle.loss(image, target)) < 1e-12, i


def test_gaussian_window_matches_opencv_and_the_reference_ssim_taps():
    g = np.load(GOLDEN)
    k = g["kernel"]
    # c_ssim_kernel of solver.cu:14-24 is the same window in float
    x = np.arange(11) - 5.0
    w = np.exp(-x * x / (2 * 1.5 ** 2))
    assert np.allclose(k, w / w.sum(), rtol=0, atol=1e-16)


@pytest.mark.parametrize("sh", [0, 3])
@pytest.mark.parametrize("size", [(9, 7), (19, 17), (33, 31)])
def test_render_reference_matches_oracle_on_renderer_test_scenes(sh, size):
    # renderer_test.cu:9-29 scenes (the reference's own bound there is 3e-5 for FP32 vs this renderer)
    need_cpu_ref()
    params = scenes.make_gaussians(7)
    cam = scenes.make_camera(*size)
    bg = [0.05, 0.1, 0.15]
    got = oracle.ref_cpu_render(params, cam, bg, sh)
    # RenderReference takes the background as float
    want = oracle.render_params(params, cam, np.float32(bg).astype(np.float64), sh)
    assert np.abs(got - want).max() < 1e-12


def test_render_reference_matches_oracle_on_single_step_scene():
    need_cpu_ref()
    params, cam = scenes.single_step_scene()
    got = oracle.ref_cpu_render(params, cam, [1, 1, 1], 3)
    want = oracle.render_params(params, cam, [1, 1, 1], 3)
    # FP64 both; depth order ties and threshold decisions could differ at
    # rounding level, neither occurs on this scene
    assert np.abs(got - want).max() < 1e-12
    target = np.clip(np.rint(oracle.render_params(scenes.random_gaussians(4096, 1), cam, [1, 1, 1], 3) * 255),
                     0, 255).astype(np.uint8)
    assert abs(oracle.ref_cpu_loss(got, target) - oracle.loss(got, target)) < 1e-12
