"""Generates tests/golden/cv_loss_golden.npz: inputs and outputs of OpenCV's own
getGaussianKernel(11, 1.5) and of the loss of the reference's CPU reference
(test/cpu_reference.h ComputeLoss: 0.8 L1 + 0.2 (1 - SSIM) with sepFilter2D,
zero border) evaluated with the real OpenCV Python module, on small seeded
images. The CPU tests compare the OpenCV shim build of cpu_reference.h
against it, so the shim is pinned to OpenCV without OpenCV at test time.

Run where cv2 is importable:  python tests/golden/make_cv_loss_golden.py
"""
import os

import cv2
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def cv_loss(image, target):
    """ComputeLoss (cpu_reference.h:118-152) with OpenCV's own filters."""
    prediction = image.astype(np.float64)
    reference = target.astype(np.float64) / 255.0
    k = cv2.getGaussianKernel(11, 1.5, cv2.CV_64F)

    def filt(x):
        return cv2.sepFilter2D(x, cv2.CV_64F, k, k, anchor=(-1, -1), delta=0, borderType=cv2.BORDER_CONSTANT)

    ma, mb = filt(prediction), filt(reference)
    aa, bb, ab = filt(prediction * prediction), filt(reference * reference), filt(prediction * reference)
    va, vb, cov = aa - ma * ma, bb - mb * mb, ab - ma * mb
    ssim = (2 * ma * mb + 0.0001) * (2 * cov + 0.0009) / ((ma * ma + mb * mb + 0.0001) * (va + vb + 0.0009))
    l1 = np.abs(prediction - reference)
    count = 3.0 * image.shape[0] * image.shape[1]
    return 0.8 * l1.sum() / count + 0.2 * (1 - ssim.sum() / count)


def main():
    rng = np.random.default_rng(2024)
    sizes = [(7, 9), (23, 37), (40, 32), (17, 64)]
    out = {"kernel": cv2.getGaussianKernel(11, 1.5, cv2.CV_64F).reshape(-1)}
    for i, (h, w) in enumerate(sizes):
        image = rng.uniform(-0.1, 1.2, size=(h, w, 3))
        target = rng.integers(0, 256, size=(h, w, 3), dtype=np.uint8)
        loss = cv_loss(image, target)
        out[f"image{i}"], out[f"target{i}"] = image, target
        out[f"loss{i}"] = np.float64(loss)
    out["cases"] = np.int64(len(sizes))
    out["cv2_version"] = np.array(cv2.__version__)
    np.savez_compressed(os.path.join(HERE, "cv_loss_golden.npz"), **out)


if __name__ == "__main__":
    main()
