"""Seeded synthetic scenes and cameras for the 3DGS training hot path.

The public datasets of the reference's benchmark are not used; these generators
produce the synthetic workloads instead:

* ``make_gaussians`` / ``make_camera`` follow the fixed test scenes of the
  reference's test support (test/test_support.h:113-148).
* ``random_gaussians`` draws the seeded distribution of the 4,096-Gaussian
  single-step case: means N(0, sigma^2) per axis, log-scales N(-3.5, 0.5^2),
  axis-angle rotations with a uniform direction and angle U(0, pi), opacity
  logits N(0, 1), SH DC N(0.5, 0.2^2) and higher bands N(0, 0.05^2).
* ``ring_cameras`` places pinhole cameras on a ring around the origin, alternating
  between +/- the given elevation, as the multi-view training scenes use.

Parameters are returned as a (58, N) float32 SoA array: row r holds field r of
every Gaussian (rows 0-2 position, 3-5 log-scale, 6-8 axis-angle, 9 opacity
logit, 10 + c * 16 + k SH coefficient k of channel c).
"""
import math

import numpy as np

from gsn import Camera

SH_C0 = 0.28209479177387814
FLT_MAX = float(np.finfo(np.float32).max)


def make_camera(width, height, fx=20.0, fy=21.0, near=0.2, far=100.0):
    """Identity-pose pinhole camera with centre ((w-1)/2, (h-1)/2)."""
    cam = Camera()
    cam.width, cam.height = width, height
    cam.fx, cam.fy = fx, fy
    cam.cx, cam.cy = 0.5 * (width - 1), 0.5 * (height - 1)
    for k in range(9):
        cam.R_c_w[k] = 1.0 if k in (0, 4, 8) else 0.0
    for k in range(3):
        cam.t_c_w[k] = 0.0
    cam.near_depth, cam.far_depth = near, far
    cam.tile_count_x = (width + 15) // 16
    cam.tile_count_y = (height + 15) // 16
    cam.pixel_offset = 0
    cam.tile_offset = 0
    return cam


def set_pose(cam, R, t):
    for k in range(9):
        cam.R_c_w[k] = float(R.reshape(-1)[k])
    for k in range(3):
        cam.t_c_w[k] = float(t[k])
    return cam


def look_at(center, target=(0.0, 0.0, 0.0), up=(0.0, 0.0, 1.0)):
    """World->camera rotation (rows right, down, forward) and translation."""
    c = np.asarray(center, dtype=np.float64)
    f = np.asarray(target, dtype=np.float64) - c
    f /= np.linalg.norm(f)
    u = np.asarray(up, dtype=np.float64)
    r = np.cross(f, u)
    if np.linalg.norm(r) < 1e-9:
        r = np.cross(f, np.array([0.0, 1.0, 0.0]))
    r /= np.linalg.norm(r)
    d = np.cross(f, r)
    R = np.stack([r, d, f]).astype(np.float32)
    t = (-R.astype(np.float64) @ c).astype(np.float32)
    return R, t


def pinhole(width, height, fx, fy, R, t, near=0.2, far=FLT_MAX):
    cam = make_camera(width, height, fx, fy, near, far)
    return set_pose(cam, R, t)


def empty_params(n):
    return np.zeros((58, n), dtype=np.float32)


def make_gaussians(count):
    """Deterministic grid of Gaussians of test/test_support.h:113-130."""
    p = empty_params(count)
    i = np.arange(count)
    p[0] = ((i % 16) - 7.5).astype(np.float32) * np.float32(0.035)
    p[1] = (((i // 16) % 16) - 7.5).astype(np.float32) * np.float32(0.035)
    p[2] = np.float32(3.0) + np.float32(0.001) * i.astype(np.float32)
    p[3], p[4], p[5] = np.log(np.float32(0.12)), np.log(np.float32(0.16)), np.log(np.float32(0.2))
    p[6], p[7], p[8] = 0.15, -0.2, 0.1
    p[9] = -1.0
    for c in range(3):
        p[10 + c * 16] = (np.float32(0.6) - np.float32(0.1) * c - np.float32(0.5)) / np.float32(SH_C0)
        for k in range(1, 16):
            p[10 + c * 16 + k] = np.float32(0.02) * np.sin((k + c + i).astype(np.float32))
    return p


def random_gaussians(count, seed, mean_sigma=1.0):
    rng = np.random.default_rng(seed)
    p = empty_params(count)
    p[0:3] = rng.normal(0.0, mean_sigma, (3, count))
    p[3:6] = rng.normal(-3.5, 0.5, (3, count))
    axis = rng.normal(size=(3, count))
    axis /= np.linalg.norm(axis, axis=0, keepdims=True)
    angle = rng.uniform(0.0, math.pi, count)
    p[6:9] = axis * angle
    p[9] = rng.normal(0.0, 1.0, count)
    for c in range(3):
        p[10 + c * 16] = rng.normal(0.5, 0.2, count)
        p[10 + c * 16 + 1:10 + c * 16 + 16] = rng.normal(0.0, 0.05, (15, count))
    return p


def single_step_scene(seed=0, count=4096):
    """4,096 Gaussians (seed 0) seen by a 128x128, fx=fy=140 camera at distance 4
    looking at the origin; the target is rendered from a seed-1 set."""
    params = random_gaussians(count, seed)
    R, t = look_at((0.0, -4.0, 0.0))
    cam = pinhole(128, 128, 140.0, 140.0, R, t)
    cam.cx = cam.cy = 63.5
    return params, cam


def ring_cameras(count, radius, elevation_deg, width, height, fx, fy, seed=None):
    cams = []
    for k in range(count):
        az = 2.0 * math.pi * k / count
        el = math.radians(elevation_deg if k % 2 == 0 else -elevation_deg)
        c = (radius * math.cos(el) * math.cos(az), radius * math.cos(el) * math.sin(az), radius * math.sin(el))
        R, t = look_at(c)
        cams.append(pinhole(width, height, fx, fy, R, t))
    return cams


MULTIVIEW_SIZES = ((640, 480), (1280, 720), (1600, 1064), (2048, 1360), (2560, 1440))


def multiview_cameras(count=32, seed=23, radius=10.0, sizes=MULTIVIEW_SIZES):
    """Views of uneven resolution: sizes drawn uniformly from `sizes`, positions
    uniform on a sphere of `radius` looking at the origin, fx = fy = 0.875 * width
    (the 1600-pixel ring cameras' 1400 / 1600)."""
    rng = np.random.default_rng(seed)
    cams = []
    for _ in range(count):
        w, h = sizes[int(rng.integers(0, len(sizes)))]
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        R, t = look_at(radius * d)
        cams.append(pinhole(w, h, 0.875 * w, 0.875 * w, R, t))
    return cams


def training_scene_cameras(count=200, held_out_every=10):
    """Ring of 200 cameras, radius 8, elevation +/-15 deg, 1600x1064, fx=fy=1400;
    every tenth camera is held out (180 train / 20 test)."""
    cams = ring_cameras(count, 8.0, 15.0, 1600, 1064, 1400.0, 1400.0)
    train = [c for k, c in enumerate(cams) if k % held_out_every != held_out_every - 1]
    test = [c for k, c in enumerate(cams) if k % held_out_every == held_out_every - 1]
    return train, test


def two_ring_cameras(count=300, radii=(8.0, 12.0), width=2048, height=1360, focal=1800.0):
    """The large scene's cameras: `count` views split over two rings of radii
    8 and 12 around the origin at elevation +/-15 deg, 2048x1360, fx = fy =
    1800."""
    half = count // 2
    return (ring_cameras(half, radii[0], 15.0, width, height, focal, focal) +
            ring_cameras(count - half, radii[1], 15.0, width, height, focal, focal))


def initial_points(target_params, count, seed, jitter=0.05):
    """`count` target means jittered by N(0, jitter^2) with the target's SH-DC colour."""
    rng = np.random.default_rng(seed)
    n = target_params.shape[1]
    pick = rng.choice(n, size=count, replace=False)
    pts = target_params[0:3, pick].T.astype(np.float64) + rng.normal(0.0, jitter, (count, 3))
    colors = np.stack([SH_C0 * target_params[10 + c * 16, pick] + 0.5 for c in range(3)], axis=1)
    return pts.astype(np.float32), np.clip(colors, 0.0, 1.0).astype(np.float32)


def params_from_points(points, colors, mean_dist2, opacity_logit=-2.2):
    """Initial Gaussians from a point cloud (gaussian_splatting.cpp:96-128):
    log-scale 0.5*log(max(d2, 1e-7)), SH DC (c - 0.5) / C0, identity rotation."""
    n = points.shape[0]
    p = empty_params(n)
    p[0:3] = points.T
    scale = 0.5 * np.log(np.maximum(mean_dist2.astype(np.float32), np.float32(1e-7)))
    p[3:6] = scale[None, :]
    for c in range(3):
        p[10 + c * 16] = (colors[:, c] - np.float32(0.5)) / np.float32(SH_C0)
    p[9] = opacity_logit
    return p
