"""Fast blend arithmetic (Renderer::SetFastBlend): the Gaussian power in Horner
form with hoisted per-record terms, the hardware exp2 approximation and depth
order on 24-bit keys. The image stays within float rounding of the reference
arithmetic's except where near-equal depths swap, the backward follows the
renderer's setting, and training matches."""
import numpy as np
import pytest

import gsn
import scenes
from helpers import dev, empty, host, sync, torch

pytestmark = pytest.mark.gpu


def _frame(fast, params, cam, target):
    t = torch()
    p = dev(params)
    img = empty((cam.height, cam.width, 3), t.float32)
    r, s = gsn.Renderer(), gsn.Solver()
    r.set_fast_blend(fast)
    assert r.render(p.data_ptr(), params.shape[1], cam, [0.2, 0.3, 0.4], img.data_ptr(), 3) == 0
    tgt = dev(target)
    s.image_gradients(cam, img.data_ptr(), tgt.data_ptr())
    ptr = s.screen_gradients(cam, r, img.data_ptr(), p.data_ptr(), params.shape[1])
    sync()
    return img.cpu().numpy(), host(ptr, np.float32, 12 * params.shape[1]).reshape(-1, 12)


@pytest.mark.parametrize("culled", [False, True])
def test_fast_blend_matches_reference_arithmetic(culled):
    params = scenes.random_gaussians(40000, 12, mean_sigma=3.0)
    cam = scenes.ring_cameras(8, 8.0, 15.0, 480, 360, 420.0, 420.0)[2]
    target = np.random.default_rng(3).integers(0, 256, size=(cam.height, cam.width, 3), dtype=np.uint8)
    exact_img, exact_g = _frame(False, params, cam, target)
    fast_img, fast_g = _frame(True, params, cam, target)
    # the fast form also orders depths on 24-bit keys: Gaussians whose depths
    # agree to 2^-16 relative may swap their blend order, which moves a few
    # pixels by up to ~1e-2; everything else moves by float rounding
    diff = np.abs(fast_img - exact_img)
    assert diff.mean() < 1e-5 and np.mean(diff > 1e-4) < 1e-3 and diff.max() < 5e-2
    scale = np.abs(exact_g[:, :11]).max(axis=0, keepdims=True)
    bad = np.abs(fast_g[:, :11] - exact_g[:, :11]) > 1e-3 * np.abs(exact_g[:, :11]) + 1e-4 * scale
    assert bad.any(axis=1).mean() < 5e-3


def test_training_with_fast_blend():
    import test_trainer_gpu as tt
    cams, images, points, colors = tt.ring_scene()
    res = []
    for fast in (0, 1):
        opts = gsn.TrainingOptions.defaults(densify_from=100000, densify_until=100, fast_blend=fast)
        tr = gsn.Trainer()
        assert tr.initialize(cams, images, points, colors, opts) == 0
        assert tr.train(400) == 0
        res.append(tr.evaluate_metrics(cams, images)["psnr"])
    assert abs(res[0] - res[1]) < 0.02


def test_fast_ssim_moments_match_exact_kernel():
    """The fast forms' SSIM gradient (products formed once per input) against the
    reference-order kernel on the same render: float-rounding agreement."""
    t = torch()
    params = scenes.random_gaussians(30000, 14, mean_sigma=3.0)
    cam = scenes.ring_cameras(8, 8.0, 15.0, 400, 300, 350.0, 350.0)[1]
    target = dev(np.random.default_rng(6).integers(0, 256, size=(cam.height, cam.width, 3), dtype=np.uint8))
    grads = []
    for fast in (False, True):
        p = dev(params)
        img = empty((cam.height, cam.width, 3), t.float32)
        r, s = gsn.Renderer(), gsn.Solver()
        r.set_fast_blend(fast)
        s.set_compute_loss(True)
        assert r.render(p.data_ptr(), params.shape[1], cam, [0, 0, 0], img.data_ptr(), 3) == 0
        # one full iteration: Iterate picks the SSIM form from the renderer
        assert s.iterate(cam, r, img.data_ptr(), target.data_ptr(), p.data_ptr(), params.shape[1], 1e-4, 3) == 0
        sync()
        grads.append((s.loss()[0], p.cpu().numpy()))
    assert abs(grads[0][0] - grads[1][0]) < 1e-5 * abs(grads[0][0]) + 1e-9
    moved = np.abs(grads[0][1] - params)
    assert np.mean(np.abs(grads[1][1] - grads[0][1]) <= 1e-3 * moved + 1e-7) > 0.999
