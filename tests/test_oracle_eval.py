"""The oracle's held-out-view metrics (RGB clamped to [0, 1], PSNR of the RGB
MSE, 11x11 Gaussian SSIM with sigma 1.5 and zero padding, mean L1) against an
independent numpy/scipy restatement."""
import numpy as np
import pytest
from scipy import ndimage

import oracle


def _window():
    d = np.arange(11) - 5.0
    g = np.exp(-d * d / (2 * 1.5 ** 2))
    return g / g.sum()


def _metrics(image, target):
    a = np.clip(image.astype(np.float64), 0, 1)
    b = target.astype(np.float64) / 255.0
    g = _window()

    def blur(x):
        x = ndimage.correlate1d(x, g, axis=1, mode="constant")
        return ndimage.correlate1d(x, g, axis=0, mode="constant")

    ssim = []
    for c in range(3):
        x, y = a[..., c], b[..., c]
        mx, my = blur(x), blur(y)
        vx, vy, cxy = blur(x * x) - mx * mx, blur(y * y) - my * my, blur(x * y) - mx * my
        ssim.append((2 * mx * my + 1e-4) * (2 * cxy + 9e-4) / ((mx * mx + my * my + 1e-4) * (vx + vy + 9e-4)))
    mse = np.mean((a - b) ** 2)
    return -10 * np.log10(mse), np.mean(ssim), np.mean(np.abs(a - b)), mse


@pytest.mark.parametrize("shape", [(1, 1), (9, 7), (40, 61)])
def test_eval_metrics_match_independent_restatement(shape):
    rng = np.random.default_rng(sum(shape))
    image = rng.uniform(-0.2, 1.2, size=shape + (3,))
    target = rng.integers(0, 256, size=shape + (3,), dtype=np.uint8)
    got = oracle.eval_metrics(image, target)
    want = _metrics(image, target)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-13)


def test_eval_metrics_identical_image():
    rng = np.random.default_rng(1)
    target = rng.integers(0, 256, size=(12, 20, 3), dtype=np.uint8)
    psnr, ssim, l1, mse = oracle.eval_metrics(target / 255.0, target)
    assert psnr == np.inf and mse == 0 and l1 == 0
    assert ssim == pytest.approx(1.0, abs=1e-14)


def test_eval_metrics_clamp():
    # values outside [0, 1] are clamped before any metric
    target = np.full((8, 8, 3), 255, np.uint8)
    psnr, ssim, l1, mse = oracle.eval_metrics(np.full((8, 8, 3), 1.7), target)
    assert mse == 0 and l1 == 0
