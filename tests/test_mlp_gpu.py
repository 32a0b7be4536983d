"""Learned density policy MLP: the GPU's fused training kernels against the
FP64 oracle's gradient, training on the GPU recovering a decision rule, and
inference with the confidence fallback."""
import numpy as np
import pytest

import gsn
import oracle
from helpers import dev, empty, host, sync, torch

pytestmark = pytest.mark.gpu


def samples(n, seed):
    rng = np.random.default_rng(seed)
    f = np.zeros((n, 16), np.float32)
    f[:, 0] = rng.exponential(1.0, n)          # mean gradient / threshold
    f[:, 1] = f[:, 0] * rng.uniform(1, 4, n)   # abs gradient / threshold
    f[:, 2] = np.log1p(rng.integers(0, 100, n))
    f[:, 3] = rng.uniform(0, 1, n)             # opacity
    f[:, 4] = np.log(f[:, 3] / (1 - f[:, 3] + 1e-6) + 1e-6)
    f[:, 5] = rng.normal(0, 1.5, n)            # log(max scale / split threshold)
    f[:, 6:13] = rng.normal(0, 1, (n, 7))
    clone = (f[:, 0] >= 1) & (f[:, 5] <= 0)
    split = (f[:, 1] >= 1) & (f[:, 5] > 0)
    prune = f[:, 3] < 0.05
    f[:, 13], f[:, 14], f[:, 15] = clone, split, prune
    labels = np.where(prune, 3, np.where(split, 2, np.where(clone, 1, 0))).astype(np.int32)
    weights = rng.uniform(0.5, 2.0, n).astype(np.float32)
    return f, labels, weights


def test_gpu_gradients_match_fp64_oracle():
    f, labels, w = samples(3000, 1)
    mlp = gsn.Mlp(seed=4)
    wts = mlp.weights()
    fd, ld, wd = dev(f), dev(labels), dev(w)
    g, loss = mlp.gradients(fd.data_ptr(), ld.data_ptr(), wd.data_ptr(), len(labels))
    # the kernels compute with the fp16 working copy of the weights
    w16 = wts.astype(np.float16).astype(np.float64)
    lref, gref = oracle.mlp_loss_gradient(w16, f, labels, w)
    assert abs(loss - lref) <= 1e-5 * abs(lref)
    assert np.max(np.abs(g - gref)) <= 1e-4 * np.max(np.abs(gref)) + 1e-7


def test_gpu_training_recovers_the_decision_rule():
    f, labels, w = samples(40000, 2)
    mlp = gsn.Mlp(seed=5)
    fd, ld, wd = dev(f), dev(labels), dev(w)
    loss0 = mlp.train(fd.data_ptr(), ld.data_ptr(), wd.data_ptr(), len(labels), 1, 3e-3)
    loss = mlp.train(fd.data_ptr(), ld.data_ptr(), wd.data_ptr(), len(labels), 400, 3e-3)
    assert loss < 0.2 * loss0
    t = torch()
    act = empty((len(labels),), t.int8)
    mlp.infer(fd.data_ptr(), len(labels), 0.0, act.data_ptr())
    sync()
    acc = np.mean(act.cpu().numpy() == labels)
    assert acc > 0.97, acc
    # with a confidence threshold of 1.01 nothing is confident: all fall back to the rule
    mlp.infer(fd.data_ptr(), len(labels), 1.01, act.data_ptr())
    sync()
    assert np.all(act.cpu().numpy() == -1)
