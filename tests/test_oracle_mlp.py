"""The FP64 restatement of the learned density MLP's objective against central
finite differences (pins the oracle the GPU gradients are checked against)."""
import numpy as np

import oracle


def test_mlp_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    w = rng.normal(size=5508) * 0.1
    f = rng.normal(size=(64, 16))
    labels = rng.integers(0, 4, 64)
    sw = rng.uniform(0.5, 2.0, 64)
    _, g = oracle.mlp_loss_gradient(w, f, labels, sw)
    for i in [0, 3, 1030, 1100, 2000, 5190, 5250, 5300, 5505]:
        wp, wm = w.copy(), w.copy()
        wp[i] += 1e-6
        wm[i] -= 1e-6
        fd = (oracle.mlp_loss_gradient(wp, f, labels, sw)[0] - oracle.mlp_loss_gradient(wm, f, labels, sw)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])
