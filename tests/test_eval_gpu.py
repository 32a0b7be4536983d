"""FP64 evaluation kernel (eval.cu) against the oracle's held-out-view
metrics, and the trainer's EvaluateMetrics built on it."""
import numpy as np
import pytest

import gsn
import oracle

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


@pytest.mark.parametrize("shape", [(1, 1), (7, 13), (8, 32), (33, 95), (140, 200), (1064, 1600)])
def test_eval_kernel_matches_oracle(shape):
    t = _torch()
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    image = rng.uniform(-0.2, 1.2, size=shape + (3,)).astype(np.float32)
    target = rng.integers(0, 256, size=shape + (3,), dtype=np.uint8)
    di, dt = t.from_numpy(image).cuda(), t.from_numpy(target).cuda()
    got = gsn.eval_metrics(di.data_ptr(), dt.data_ptr(), shape[1], shape[0])
    psnr, ssim, l1, mse = oracle.eval_metrics(image.astype(np.float64), target)
    # FP64 on both sides; only the summation order (and FMA contraction)
    # differs: the oracle's sequential sum over 5.1M terms carries up to
    # ~n * 2^-53 relative error, hence rel 1e-10
    assert got["psnr"] == pytest.approx(psnr, abs=1e-9)
    assert got["ssim"] == pytest.approx(ssim, rel=1e-10, abs=1e-12)
    assert got["l1"] == pytest.approx(l1, rel=1e-10, abs=1e-12)
    assert got["mse"] == pytest.approx(mse, rel=1e-10)
    # fixed-order reduction: bit-identical on a repeat
    again = gsn.eval_metrics(di.data_ptr(), dt.data_ptr(), shape[1], shape[0])
    assert again == got


def test_eval_kernel_identical_image():
    t = _torch()
    target = np.random.default_rng(3).integers(0, 256, size=(50, 70, 3), dtype=np.uint8)
    di = t.from_numpy((target / 255.0).astype(np.float32)).cuda()
    dt = t.from_numpy(target).cuda()
    got = gsn.eval_metrics(di.data_ptr(), dt.data_ptr(), 70, 50)
    # the fp32 image differs from k / 255 by at most half an ulp
    assert got["mse"] < 1e-14 and got["psnr"] > 140
    assert got["ssim"] == pytest.approx(1.0, abs=1e-9)


def test_trainer_evaluate_metrics_match_oracle():
    import test_trainer_gpu as tt
    cams, images, points, colors = tt.ring_scene(views=4, n=4000)
    tr = gsn.Trainer()
    assert tr.initialize(cams, images, points, colors) == 0
    assert tr.train(200) == 0
    m = tr.evaluate_metrics(cams, images)
    want = np.zeros(3)
    loss = 0.0
    for c, img in zip(cams, images):
        r = tt.render(tr, c).astype(np.float64)
        psnr, ssim, l1, _ = oracle.eval_metrics(r, img)
        want += [psnr, ssim, l1]
        loss += oracle.loss(r, img)
    want /= len(cams)
    assert m["psnr"] == pytest.approx(want[0], abs=1e-8)
    assert m["ssim"] == pytest.approx(want[1], abs=1e-10)
    assert m["l1"] == pytest.approx(want[2], abs=1e-10)
    assert m["loss"] == pytest.approx(loss / len(cams), abs=1e-6)
