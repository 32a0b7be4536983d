"""Scenes of the reference's solver tests (solver_test.cu) and FP64 helpers
built on the oracle: loss(params) and its analytic gradient."""
import math

import numpy as np

import oracle
import scenes


def rodrigues(axis, angle):
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + math.sin(angle) * K + (1 - math.cos(angle)) * K @ K


def differentiable_scene():
    """MakeDifferentiableScene of solver_test.cu:31-42 on a 9x7 camera."""
    cam = scenes.make_camera(9, 7)
    R = (rodrigues([0, 1, 0], 0.55) @ rodrigues([1, 0, 0], 0.35) @ rodrigues([0, 0, 1], 0.2)).astype(np.float32)
    scenes.set_pose(cam, R, np.zeros(3, np.float32))
    p = scenes.make_gaussians(1)
    p[0:3, 0] = R.T @ np.array([0.2, -0.1, 3.0], dtype=np.float32)
    p[3:6, 0] = np.log(np.array([0.6, 0.45, 0.35], dtype=np.float32))
    return p, cam, R


def overlapping_scene():
    """Three overlapping Gaussians with a coloured background (solver_test.cu:97-116)."""
    base, cam, R = differentiable_scene()
    p = scenes.make_gaussians(3)
    for i in range(3):
        p[0:3, i] = R.T @ np.array([0.2 - 0.12 * i, -0.1 + 0.09 * i, 3.0 + 0.4 * i], dtype=np.float32)
        p[3:6, i] = base[3:6, 0]
        p[9, i] = -0.4 + 0.3 * i
        for c in range(3):
            p[10 + c * 16, i] = (0.25 + 0.15 * ((i + c) % 3) - 0.5) / scenes.SH_C0
    p = np.ascontiguousarray(p[:, ::-1])
    return p, cam, [0.12, 0.31, 0.57]


def constant_target(cam, rgb=(180, 190, 200)):
    # cv::Scalar(180, 190, 200) on a CV_8UC3 Mat: channel 0 = 180, 1 = 190, 2 = 200
    t = np.zeros((cam.height, cam.width, 3), dtype=np.uint8)
    t[:] = np.array(rgb, dtype=np.uint8)
    return t


def loss_of(params, cam, target, background, sh):
    img = oracle.render_params(params, cam, background, sh)
    return oracle.loss(img, target)


def analytic(params, cam, target, background, sh):
    """FP64 oracle gradients: (g58, g9, abs2, stats, abs_stats, image)."""
    proj = oracle.project(params, cam, sh)
    offsets, ids = oracle.tile_lists(proj, cam)
    img = oracle.render(proj, cam, offsets, ids, background)[0]
    gI = oracle.loss_gradient(img, target)
    g9, a2 = oracle.backward(proj, cam, offsets, ids, img, gI)
    stats, abs_stats = oracle.projection_statistics(proj, cam, g9, a2)
    g58 = oracle.map_gradients(params, cam, sh, g9)
    return dict(g58=g58, g9=g9, a2=a2, stats=stats, abs_stats=abs_stats, image=img, image_grad=gI)


def active_fields(sh):
    k = (sh + 1) ** 2
    return [f for f in range(58) if f < 10 or (f - 10) % 16 < k]


def finite_difference(params, cam, target, background, sh, i, field, h=5e-4):
    hi = params.copy()
    lo = params.copy()
    hi[field, i] = np.float32(params[field, i] + h)
    lo[field, i] = np.float32(params[field, i] - h)
    step = float(hi[field, i]) - float(lo[field, i])
    return (loss_of(hi, cam, target, background, sh) - loss_of(lo, cam, target, background, sh)) / step
