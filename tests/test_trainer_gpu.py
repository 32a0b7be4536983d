"""GPU tests of the trainer (reference gaussian_splatting_test.cpp) through the C ABI."""
import numpy as np
import pytest

import gsn
import oracle
import scenes
from helpers import dev, empty, sync, torch

pytestmark = pytest.mark.gpu


def make_scene():
    """MakeScene of test_support.h:150-162: one 9x7 view, four points."""
    cam = scenes.make_camera(9, 7)
    cam.cx, cam.cy = 4.0, 3.0
    cam.far_depth = scenes.FLT_MAX
    image = np.zeros((7, 9, 3), dtype=np.uint8)
    image[:] = (160, 170, 180)
    points = np.array([[-0.1, -0.1, 3], [0.1, -0.1, 3], [-0.1, 0.1, 3], [0.1, 0.1, 3]], dtype=np.float32)
    colors = np.tile(np.array([0.6, 0.5, 0.4], dtype=np.float32), (4, 1))
    return cam, image, points, colors


def render(trainer, cam):
    t = torch()
    img = empty((cam.height, cam.width, 3), t.float32)
    assert trainer.render(cam, img.data_ptr()) == 0
    sync()
    return img.cpu().numpy()


def test_initializes_iterates_saves_and_reloads(tmp_path):
    cam, image, points, colors = make_scene()
    tr = gsn.Trainer()
    assert tr.initialize([cam], [image], points, colors) == 0
    before = render(tr, cam)
    assert tr.train(3) == 0
    after = render(tr, cam)
    assert np.isfinite(before).all() and np.isfinite(after).all()
    assert oracle.loss(after.astype(np.float64), image) < oracle.loss(before.astype(np.float64), image)
    path = tmp_path / "model.ply"
    assert tr.save(path) == 0
    st, params = gsn.ply_read(path)
    assert st == 0 and params.shape[1] == 4
    t = torch()
    p = dev(params)
    img = empty((7, 9, 3), t.float32)
    r = gsn.Renderer()
    assert r.render(p.data_ptr(), 4, cam, [0, 0, 0], img.data_ptr(), 0) == 0
    sync()
    assert np.abs(after - img.cpu().numpy()).max() < 2e-5


def test_crosses_density_control_boundary(tmp_path):
    cam, image, points, colors = make_scene()
    tr = gsn.Trainer()
    assert tr.initialize([cam], [image], points, colors) == 0
    assert tr.train(600) == 0
    assert np.isfinite(render(tr, cam)).all()
    path = tmp_path / "density.ply"
    assert tr.save(path) == 0
    st, params = gsn.ply_read(path)
    assert st == 0
    assert params.shape[1] == 2 * len(points)
    assert np.isfinite(params).all()


def test_rejects_empty_scene_and_supports_zero_iterations():
    tr = gsn.Trainer()
    cam, image, points, colors = make_scene()
    assert tr.initialize([], [], points, colors) != 0
    assert tr.initialize([cam], [image], points, colors) == 0
    before = render(tr, cam)
    assert tr.train(0) == 0
    after = render(tr, cam)
    assert np.array_equal(before, after)


def test_evaluate_reports_fp64_psnr():
    cam, image, points, colors = make_scene()
    tr = gsn.Trainer()
    assert tr.initialize([cam], [image], points, colors) == 0
    psnr, loss = tr.evaluate([cam], [image])
    img = render(tr, cam).astype(np.float64)
    mse = np.mean((img - image / 255.0) ** 2)
    assert abs(psnr - (-10 * np.log10(mse))) < 1e-4
    assert abs(loss - oracle.loss(img, image)) < 1e-6
