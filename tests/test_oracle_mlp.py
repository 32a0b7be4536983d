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


def test_shipped_density_policy_weights_are_well_formed():
    """The trained density policy shipped with the package (large-scene
    protocol) has the MLP's 5,508 parameters, all finite, and gives a proper
    action distribution under the FP64 oracle's forward pass."""
    import os

    import numpy as np

    import oracle
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gs-native_b200", "policies",
                        "density_mlp_large_scene.npy")
    w = np.load(path)
    assert w.dtype == np.float32 and w.shape == (5508,) and np.isfinite(w).all()
    feats = np.random.default_rng(0).normal(size=(64, 16))
    logits = oracle.mlp_forward(w, feats)[-1]
    p = np.exp(logits - logits.max(axis=1, keepdims=True))
    p /= p.sum(axis=1, keepdims=True)
    assert logits.shape == (64, 4) and np.isfinite(p).all()
