"""Batched form: a training iteration captured once as a CUDA graph and replayed
from a device schedule must train exactly like the eager Render + Iterate
sequence (up to the summation order of the backward's atomics), report record
overflow through its sticky status instead of synchronising, and leave the
Adam step counter where the eager path would."""
import numpy as np
import pytest

import gsn
import scenes
from helpers import dev, empty, host, sync, torch

pytestmark = pytest.mark.gpu

W, H = 320, 200


def views_scene(n=20000, views=4):
    cams = scenes.ring_cameras(views, 6.0, 15.0, W, H, 280.0, 280.0)
    hidden = scenes.random_gaussians(n, 11, mean_sigma=1.2)
    model = scenes.random_gaussians(n, 12, mean_sigma=1.2)
    t = torch()
    r = gsn.Renderer()
    hp = dev(hidden)
    img = empty((H, W, 3), t.float32)
    targets = empty((views, H, W, 3), t.uint8)
    for k, c in enumerate(cams):
        assert r.render(hp.data_ptr(), n, c, [0, 0, 0], img.data_ptr(), 3) == 0
        targets[k] = (img * 255.0).round().clamp(0, 255).to(t.uint8)
    sync()
    views_scene.hidden = hidden
    return cams, model, targets


def eager(cams, model, targets, views, lrs):
    t = torch()
    p = dev(model)
    img = empty((H, W, 3), t.float32)
    r, s = gsn.Renderer(), gsn.Solver()
    s.set_compute_loss(True)
    stride = H * W * 3
    for v, lr in zip(views, lrs):
        assert r.render(p.data_ptr(), p.shape[1], cams[v], [0, 0, 0], img.data_ptr(), 3) == 0
        assert s.iterate(cams[v], r, img.data_ptr(), targets.data_ptr() + v * stride, p.data_ptr(), p.shape[1], lr,
                         3) == 0
    sync()
    return p.cpu().numpy(), s.loss(), s.moments()[2]


def graph_run(cams, model, targets, views, lrs, capacity=4_000_000, chunks=1):
    t = torch()
    p = dev(model)
    img = empty((H, W, 3), t.float32)
    r, s = gsn.Renderer(), gsn.Solver()
    s.set_compute_loss(True)
    g = gsn.Graph()
    g.capture(r, s, p.data_ptr(), p.shape[1], cams, targets.data_ptr(), H * W * 3, [0, 0, 0], img.data_ptr(), 3,
              capacity)
    k = len(views) // chunks
    for c in range(chunks):
        end = len(views) if c == chunks - 1 else (c + 1) * k
        g.run(views[c * k:end], lrs[c * k:end])
    status = g.check()
    out = p.cpu().numpy(), s.loss(), s.moments()[2], status, g.launches_per_step()
    g.close()
    return out


def test_graph_replay_trains_like_eager_steps():
    cams, model, targets = views_scene()
    views = [0, 2, 1, 3, 3, 0, 1, 2]
    lrs = [1.6e-4 * (1 - 0.05 * k) for k in range(len(views))]
    pe, le, ite = eager(cams, model, targets, views, lrs)
    pg, lg, itg, status, launches = graph_run(cams, model, targets, views, lrs, chunks=2)
    assert status == 0
    assert ite == itg == len(views)
    assert launches > 10
    moved = np.abs(pe - model)
    diff = np.abs(pg - pe)
    # identical arithmetic; only the backward's atomic summation order differs
    assert np.mean(diff <= 1e-6 + 1e-3 * moved) > 0.999
    assert abs(lg[0] - le[0]) <= 1e-4 * abs(le[0])
    assert abs(lg[3] - le[3]) < 1e-3  # PSNR of the last step, dB


def test_graph_reports_record_overflow_without_faulting():
    cams, model, targets = views_scene(n=4000, views=2)
    views, lrs = [0, 1, 0], [1e-4] * 3
    *_, status, _ = graph_run(cams, model, targets, views, lrs, capacity=2000)
    assert status == -4  # GSN_ERR_CAPACITY


def test_graph_rejects_mixed_resolutions_and_bad_views():
    cams, model, targets = views_scene(n=2000, views=2)
    t = torch()
    p = dev(model)
    img = empty((H, W, 3), t.float32)
    r, s = gsn.Renderer(), gsn.Solver()
    g = gsn.Graph()
    other = scenes.ring_cameras(1, 6.0, 15.0, W + 16, H, 280.0, 280.0)[0]
    with pytest.raises(gsn.GsnError):
        g.capture(r, s, p.data_ptr(), p.shape[1], [cams[0], other], targets.data_ptr(), H * W * 3, [0, 0, 0],
                  img.data_ptr(), 3, 1_000_000)
    g.capture(r, s, p.data_ptr(), p.shape[1], cams, targets.data_ptr(), H * W * 3, [0, 0, 0], img.data_ptr(), 3,
              1_000_000)
    with pytest.raises(gsn.GsnError):
        g.run([0, 2], [1e-4, 1e-4])  # view 2 does not exist
    assert g.check() == 0
    g.close()


def _graph_vs_eager(densify_from, densify_until, iterations):
    cams, _, targets = views_scene(n=20000, views=6)
    hidden = views_scene.hidden
    imgs = [targets[k].cpu().numpy() for k in range(6)]
    points, colors = scenes.initial_points(hidden, 4000, 5)
    out = {}
    for graph in (0, 1):
        opts = gsn.TrainingOptions.defaults(densify_from=densify_from, densify_until=densify_until,
                                            densify_interval=100, sh_degree_interval=100,
                                            opacity_reset_interval=100000, graph=graph)
        tr = gsn.Trainer()
        assert tr.initialize(cams, imgs, points, colors, opts) == 0
        assert tr.train(iterations) == 0
        psnr, loss = tr.evaluate(cams, imgs)
        st = tr.state()
        out[graph] = (psnr, loss, st["count"], st["completed"])
        tr.close()
    assert out[0][3] == out[1][3] == iterations
    return out


def test_trainer_graph_steady_state_trains_like_eager():
    """Iterations after densify_until run as graph replays in the trainer; with
    the same schedule (camera order, learning rates) the result matches the
    eager trainer up to the backward's atomic summation order. Without density
    control (360 replayed steps, SH ramp included) that is the only difference;
    with it, threshold decisions amplify the float-atomic noise chaotically, so
    that run only checks the counts and a loose PSNR bound."""
    out = _graph_vs_eager(100000, 100, 460)
    assert out[0][2] == out[1][2] and abs(out[0][0] - out[1][0]) < 0.03, out
    # three runs of each, compared on their medians
    runs = [_graph_vs_eager(100, 400, 460) for _ in range(3)]
    psnr = [float(np.median([r[g][0] for r in runs])) for g in (0, 1)]
    count = [float(np.median([r[g][2] for r in runs])) for g in (0, 1)]
    assert abs(count[0] - count[1]) <= 0.01 * count[0] and abs(psnr[0] - psnr[1]) < 0.3, runs
