"""Exact tile culling (project.cu cull_row_span): the culled renderer emits a
subset of the reference's records; the image, the per-pixel work and the
gradients are unchanged; every dropped record is one whose alpha stays below
1/255 at every pixel of its tile (checked in FP64 from the device's own
projected values)."""
import numpy as np
import pytest

import gsn
import scenes
from helpers import dev, empty, gsn_sorted_lists, host, sync, torch
from test_solver_gpu import rows_close

pytestmark = pytest.mark.gpu


def _scene(n=60000, width=640, height=480, seed=8, cam_index=0):
    params = scenes.random_gaussians(n, seed, mean_sigma=3.0)
    cams = scenes.ring_cameras(8, 8.0, 15.0, width, height, 560.0, 560.0)
    return params, cams[cam_index]


def _render(params, cam, culled, bg=(0.3, 0.5, 0.7)):
    t = torch()
    p = dev(params)
    img = empty((cam.height, cam.width, 3), t.float32)
    r = gsn.Renderer()
    r.set_exact_culling(culled)
    assert r.render(p.data_ptr(), params.shape[1], cam, bg, img.data_ptr(), 3) == 0
    sync()
    return r, p, img


@pytest.mark.parametrize("cam_index", [0, 3])
def test_culled_image_identical_and_records_subset(cam_index):
    params, cam = _scene(cam_index=cam_index)
    r0, p0, img0 = _render(params, cam, False)
    r1, p1, img1 = _render(params, cam, True)
    assert torch().equal(img0, img1)
    ids0, off0 = gsn_sorted_lists(r0, cam)
    ids1, off1 = gsn_sorted_lists(r1, cam)
    assert off1[-1] < 0.9 * off0[-1]  # the synthetic scene loses >10 % of its records
    # per tile, the culled list is an ordered subsequence of the full list
    for t in range(cam.tile_count_x * cam.tile_count_y):
        full = ids0[off0[t]:off0[t + 1]]
        cut = ids1[off1[t]:off1[t + 1]]
        keep = np.isin(full, cut)
        assert np.array_equal(full[keep], cut)
    # the visibility statistic keeps the rectangle counts
    b0, b1 = r0.buffers(), r1.buffers()
    n = params.shape[1]
    assert np.array_equal(host(b0.tile_counts, np.int32, n), host(b1.tile_counts, np.int32, n))


def test_dropped_records_never_reach_alpha_threshold():
    params, cam = _scene(n=30000, width=320, height=240)
    r0, _, _ = _render(params, cam, False)
    r1, _, _ = _render(params, cam, True)
    ids0, off0 = gsn_sorted_lists(r0, cam)
    ids1, off1 = gsn_sorted_lists(r1, cam)
    b = r1.buffers()
    n = params.shape[1]
    means = host(b.means, np.float32, 2 * n).reshape(n, 2).astype(np.float64)
    conic = host(b.conic_opacity, np.float32, 4 * n).reshape(n, 4).astype(np.float64)
    ys, xs = np.mgrid[0:16, 0:16]
    worst = 0.0
    dropped = 0
    for t in range(cam.tile_count_x * cam.tile_count_y):
        full = ids0[off0[t]:off0[t + 1]]
        gone = full[~np.isin(full, ids1[off1[t]:off1[t + 1]])]
        if not len(gone):
            continue
        dropped += len(gone)
        tx, ty = t % cam.tile_count_x, t // cam.tile_count_x
        px = (tx * 16 + xs).ravel()[None, :]
        py = (ty * 16 + ys).ravel()[None, :]
        dx = px - means[gone, 0:1]
        dy = py - means[gone, 1:2]
        a, bb, c, o = (conic[gone, k:k + 1] for k in range(4))
        alpha = o * np.exp(-0.5 * (a * dx * dx + c * dy * dy) - bb * dx * dy)
        worst = max(worst, float(alpha.max()))
    assert dropped > 1000
    assert worst < 1.0 / 255.0


def test_culled_gradients_match():
    params, cam = _scene(n=40000, width=480, height=360)
    target = np.random.default_rng(2).integers(0, 256, size=(cam.height, cam.width, 3), dtype=np.uint8)
    out = []
    for culled in (False, True):
        r, p, img = _render(params, cam, culled, bg=(0, 0, 0))
        s = gsn.Solver()
        tgt = dev(target)
        s.image_gradients(cam, img.data_ptr(), tgt.data_ptr())
        ptr = s.screen_gradients(cam, r, img.data_ptr(), p.data_ptr(), params.shape[1])
        sync()
        out.append(host(ptr, np.float32, 12 * params.shape[1]).reshape(-1, 12))
    ok, where = rows_close(out[1][:, :11].T, out[0][:, :11].T, rel=2e-4, floor=2e-5)
    assert ok, where


def _train(culled, iterations, densify_until):
    import test_trainer_gpu as tt
    cams, images, points, colors = tt.ring_scene()
    opts = gsn.TrainingOptions.defaults(densify_from=100, densify_until=densify_until, densify_interval=100,
                                        exact_culling=culled)
    tr = gsn.Trainer()
    assert tr.initialize(cams, images, points, colors, opts) == 0
    assert tr.train(iterations) == 0
    return tr.evaluate_metrics(cams, images)["psnr"], tr.state()["count"]


def test_training_with_culling_matches_plain():
    # without density control the runs differ only by float-atomic order
    a, b = _train(0, 400, 0), _train(1, 400, 0)
    assert a[1] == b[1] and abs(a[0] - b[0]) < 0.02
    # with density control, threshold decisions amplify that noise chaotically:
    # plain runs of this 10-view scene spread by up to ~0.3 dB from one process
    # to the next, and their Gaussian counts by about 1 %, so only loose bounds
    # are meaningful here
    # so each form is run three times and compared on its medians
    runs = {culled: [_train(culled, 900, 700) for _ in range(3)] for culled in (0, 1)}
    p = [float(np.median([r[k] for r in runs[0]])) for k in (0, 1)]
    c = [float(np.median([r[k] for r in runs[1]])) for k in (0, 1)]
    assert abs(c[0] - p[0]) < 0.35, runs
    assert abs(c[1] - p[1]) <= 0.03 * p[1], runs
