"""Error of the plain FP32 form and of the precision form (bf16 SH storage,
tensor-core SSIM, FP64 near-singular conics) against the FP64 oracle on the
single-step scene (4,096 Gaussians, 128 x 128, SH degree 3, white background),
for the image, the loss and each gradient tensor. Both forms get the same
parameters with their SH rounded to bf16, so the figures are the arithmetic
error of each form; the storage rounding itself is reported separately.
Run with -s to print the table.

Measured on B200 (max / mean relative to max |ref|): plain image 1.4e-6 /
1.1e-7, loss 9.4e-8, dL/dI 2.0e-5 / 1.1e-6, screen gradients 1.6e-5 / 9.8e-8,
parameter gradients 5.3e-6 / 1.4e-8; precision image 1.4e-6 / 1.1e-7, loss
1.1e-4, dL/dI 1.3e-3 / 5.5e-5, screen gradients 9.7e-4 / 5.6e-6, parameter
gradients 3.7e-4 / 7.3e-7; bf16 storage of the SH changes the image by up to
7.2e-4."""
import numpy as np
import pytest

import gsn
import oracle
import scenes
from helpers import dev, empty, host, sync, torch

pytestmark = pytest.mark.gpu


def rounded(params):
    t = torch()
    out = params.copy()
    out[10:] = t.from_numpy(params[10:]).to(t.bfloat16).float().numpy()
    return out


def run_form(params, cam, target, precision):
    t = torch()
    n = params.shape[1]
    r, s = gsn.Renderer(), gsn.Solver()
    if precision:
        r.set_bf16_sh(True)
        s.set_bf16_sh(True)
    s.set_compute_loss(True)
    p = gsn.to_precision_layout(params, t) if precision else dev(params)
    img = empty((cam.height, cam.width, 3), t.float32)
    assert r.render(p.data_ptr(), n, cam, [1, 1, 1], img.data_ptr(), 3) == 0
    gi = s.image_gradients(cam, img.data_ptr(), target.data_ptr())
    sync()
    out = dict(image=img.cpu().numpy(), loss=s.loss()[0],
               image_grad=host(gi, np.float32, cam.height * cam.width * 3).reshape(cam.height, cam.width, 3))
    sp = s.screen_gradients(cam, r, img.data_ptr(), p.data_ptr(), n)
    sync()
    out["screen"] = host(sp, np.float32, 12 * n).reshape(n, 12)[:, :9].T
    g = empty((58, n), t.float32)
    s.map_gradients(cam, r, p.data_ptr(), n, 3, g.data_ptr())
    sync()
    out["mapped"] = g.cpu().numpy()
    return out


def errors(mine, ref):
    scale = max(float(np.max(np.abs(ref))), 1e-30)
    d = np.abs(np.asarray(mine, np.float64) - ref)
    return float(np.max(d)) / scale, float(np.mean(d)) / scale


def test_error_against_fp64_oracle_is_stated_and_bounded():
    params, cam = scenes.single_step_scene()
    params = rounded(params)
    tp = scenes.random_gaussians(4096, 1)
    timg = oracle.render_params(tp, cam, [1, 1, 1], 3)
    target_np = np.clip(np.rint(timg * 255), 0, 255).astype(np.uint8)
    target = dev(target_np)
    # FP64 oracle on the same (bf16-rounded) parameters
    proj = oracle.project(params, cam, 3)
    offsets, ids = oracle.tile_lists(proj, cam)
    img64 = oracle.render(proj, cam, offsets, ids, [1, 1, 1])[0]
    loss64 = oracle.loss(img64, target_np)
    gi64 = oracle.loss_gradient(img64, target_np)
    g9, _ = oracle.backward(proj, cam, offsets, ids, img64, gi64)
    g58 = oracle.map_gradients(params, cam, 3, g9)
    table = {}
    for name, precision in (("plain_fp32", False), ("precision_bf16", True)):
        f = run_form(params, cam, target, precision)
        table[name] = {
            "image": errors(f["image"], img64),
            "loss": (abs(f["loss"] - loss64) / abs(loss64),) * 2,
            "image_grad": errors(f["image_grad"], gi64),
            "screen_grad": errors(f["screen"], g9),
            "mapped_grad": errors(f["mapped"], g58),
        }
    # storage rounding: fp32 SH against bf16-rounded SH, plain renderer
    raw, _ = scenes.single_step_scene()
    img_fp32 = run_form(raw, cam, target, False)["image"]
    storage = float(np.max(np.abs(img_fp32 - img64)))
    print("\nerror vs FP64 oracle (max / mean of |err|, relative to max |ref|):")
    for name, rows in table.items():
        for k, (mx, mn) in rows.items():
            print(f"  {name:15s} {k:12s} max {mx:.3e}  mean {mn:.3e}")
    print(f"  bf16 SH storage rounding: max image change {storage:.3e}")
    plain, prec = table["plain_fp32"], table["precision_bf16"]
    assert plain["image"][0] < 1e-4 and prec["image"][0] < 1e-4
    assert plain["loss"][0] < 1e-5 and prec["loss"][0] < 3e-4
    assert plain["image_grad"][0] < 1e-4 and prec["image_grad"][0] < 2e-3
    assert plain["screen_grad"][1] < 1e-3 and prec["screen_grad"][1] < 2e-3
    assert plain["mapped_grad"][1] < 1e-3 and prec["mapped_grad"][1] < 2e-3


def ring_scene(width=400, height=266):
    """The config-1 ring scene at quarter resolution (fx = fy = 350, the
    1600x1064 cameras' 1400 scaled): hidden 1.5M-Gaussian model (seed 7),
    100k initial points (target means jittered, target DC colours, 3-NN
    scales, opacity logit -2.2)."""
    train, _ = scenes.training_scene_cameras()
    for c in train:
        c.width, c.height = width, height
        c.fx, c.fy = c.fx * width / 1600.0, c.fy * height / 1064.0
        c.cx, c.cy = 0.5 * (width - 1), 0.5 * (height - 1)
        c.tile_count_x, c.tile_count_y = (width + 15) // 16, (height + 15) // 16
    hidden = scenes.random_gaussians(1_500_000, 7, mean_sigma=3.0)
    points, colors = scenes.initial_points(hidden, 100_000, 3)
    d2, _ = gsn.knn3_host(points)
    params = scenes.params_from_points(points, colors, d2)
    return train, hidden, params


def test_error_over_ten_seeded_iterations_of_the_ring_scene():
    """Error of each form against the FP64 oracle over 10 seeded training
    iterations of the config-1 scene (quarter resolution; SH degree 3 from the
    start, the higher bands seeded with N(0, 0.02^2) so every gradient row is
    exercised; views drawn with seed 2 from the 180 training views). At every
    iteration the oracle evaluates the form's own current parameters, so the
    figures are the form's arithmetic error, accumulated as the worst max and
    the worst mean over the 10 iterations. Run with -s to print the table."""
    t = torch()
    train, hidden, params = ring_scene()
    rng = np.random.default_rng(2)
    for c in range(3):
        params[11 + 16 * c:26 + 16 * c] = rng.normal(0.0, 0.02, (15, params.shape[1]))
    params = rounded(params)
    n = params.shape[1]
    views = rng.choice(len(train), 10, replace=False)
    hp = dev(hidden)
    targets = {}
    for v in views:
        cam = train[v]
        img = empty((cam.height, cam.width, 3), t.float32)
        assert gsn.Renderer().render(hp.data_ptr(), hp.shape[1], cam, [0, 0, 0], img.data_ptr(), 3) == 0
        targets[v] = (img * 255.0).round().clamp(0, 255).to(t.uint8)
    del hp
    sync()
    table = {}
    for name, precision in (("plain_fp32", False), ("precision_bf16", True)):
        r, s = gsn.Renderer(), gsn.Solver()
        if precision:
            r.set_bf16_sh(True)
            s.set_bf16_sh(True)
        s.set_compute_loss(True)
        p = gsn.to_precision_layout(params, t) if precision else dev(params)
        worst = {}
        for k, v in enumerate(views):
            cam, target = train[v], targets[v]
            img = empty((cam.height, cam.width, 3), t.float32)
            assert r.render(p.data_ptr(), n, cam, [0, 0, 0], img.data_ptr(), 3) == 0
            gi = s.image_gradients(cam, img.data_ptr(), target.data_ptr())
            sync()
            image, loss = img.cpu().numpy(), s.loss()[0]
            image_grad = host(gi, np.float32, cam.pixels * 3).reshape(cam.height, cam.width, 3)
            sp = s.screen_gradients(cam, r, img.data_ptr(), p.data_ptr(), n)
            sync()
            screen = host(sp, np.float32, 12 * n).reshape(n, 12)[:, :9].T
            g = empty((58, n), t.float32)
            s.map_gradients(cam, r, p.data_ptr(), n, 3, g.data_ptr())
            sync()
            mapped = g.cpu().numpy()
            # FP64 oracle on this iteration's parameters
            cur = (gsn.from_precision_layout(p, n, t) if precision else p).cpu().numpy()
            target_np = target.cpu().numpy()
            proj = oracle.project(cur, cam, 3)
            offsets, ids = oracle.tile_lists(proj, cam)
            img64 = oracle.render(proj, cam, offsets, ids, [0, 0, 0])[0]
            loss64 = oracle.loss(img64, target_np)
            gi64 = oracle.loss_gradient(img64, target_np)
            g9, _ = oracle.backward(proj, cam, offsets, ids, img64, gi64)
            g58 = oracle.map_gradients(cur, cam, 3, g9)
            errs = {"image": errors(image, img64), "loss": (abs(loss - loss64) / abs(loss64),) * 2,
                    "image_grad": errors(image_grad, gi64), "screen_grad": errors(screen, g9),
                    "mapped_grad": errors(mapped, g58)}
            for key, (mx, mn) in errs.items():
                a, b = worst.get(key, (0.0, 0.0))
                worst[key] = (max(a, mx), max(b, mn))
            # the training step itself (the schedule's position learning rate at iteration k + 1)
            lr = 1.6e-4 * 1.1 * 8.0 * (1.6e-6 / 1.6e-4) ** ((k + 1) / 30000.0)
            assert s.iterate(cam, r, img.data_ptr(), target.data_ptr(), p.data_ptr(), n, lr, 3) == 0
        sync()
        table[name] = worst
    print("\nworst error over 10 iterations vs FP64 oracle (max / mean of |err|, relative to max |ref|):")
    for name, rows in table.items():
        for key, (mx, mn) in rows.items():
            print(f"  {name:15s} {key:12s} max {mx:.3e}  mean {mn:.3e}")
    # Bounds from the B200 measurement (worst max / worst mean over the 10
    # iterations; plain then precision): image 5.3e-4 / 3.7e-7 and 5.2e-4 /
    # 3.7e-7 - both forms' maxima are FP32-vs-FP64 flips of the 1/255 and 1e-4
    # thresholds on a few pixels; loss 3.2e-5 and 3.1e-3 (the tensor-core
    # SSIM's hi/lo bf16 products lose the variance terms' cancellation);
    # dL/dI mean 1.6e-5 and 2.8e-4, its maxima (0.24, 0.23) are L1 sign flips
    # where |I - T| is at rounding level; screen gradients 6.9e-5 / 2.4e-9 and
    # 1.5e-3 / 5.4e-8; parameter gradients 7.3e-5 / 3.3e-9 and 1.8e-3 / 7.1e-8.
    plain, prec = table["plain_fp32"], table["precision_bf16"]
    assert plain["image"][0] < 2e-3 and prec["image"][0] < 2e-3
    assert plain["image"][1] < 1e-6 and prec["image"][1] < 1e-6
    assert plain["loss"][0] < 1e-4 and prec["loss"][0] < 1e-2
    assert plain["image_grad"][1] < 1e-4 and prec["image_grad"][1] < 1e-3
    assert plain["screen_grad"][0] < 1e-3 and prec["screen_grad"][0] < 1e-2
    assert plain["screen_grad"][1] < 1e-6 and prec["screen_grad"][1] < 1e-6
    assert plain["mapped_grad"][0] < 1e-3 and prec["mapped_grad"][0] < 1e-2
    assert plain["mapped_grad"][1] < 1e-6 and prec["mapped_grad"][1] < 1e-6
