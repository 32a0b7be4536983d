"""COLMAP scene loader and image writers (CPU): the binary readers, name sort,
every-8th test split, intrinsics scaling with the half-pixel shift, quaternion
to rotation, area downscale, point cloud, error cases, and the PNG writer
(decoded here with zlib). Mirrors the reference's ReadColmapScene
(src/io/data_io.cpp:328-418) without OpenCV."""
import numpy as np
import pytest

import colmap_writer as cw
import gsn


def _random_views(rng, count, width, height):
    names = [f"img_{k:03d}.jpg" for k in rng.permutation(count)]
    views = []
    for name in names:
        q = rng.normal(size=4)
        views.append({"name": name, "qvec": q / np.linalg.norm(q), "tvec": rng.normal(size=3),
                      "image": rng.integers(0, 256, size=(height, width, 3), dtype=np.uint8)})
    return views


def _scene(tmp_path, rng, count=19, width=48, height=32, points=50):
    views = _random_views(rng, count, width, height)
    pts = rng.normal(size=(points, 3))
    cols = rng.integers(0, 256, size=(points, 3))
    cw.write_scene(str(tmp_path), width, height, 40.0, 42.0, 23.5, 15.25, views, pts, cols)
    return views, pts, cols


def test_reads_scene_split_and_cameras(tmp_path):
    rng = np.random.default_rng(3)
    views, pts, cols = _scene(tmp_path, rng)
    s = gsn.ColmapScene(tmp_path)
    ordered = sorted(views, key=lambda v: v["name"])
    test = [v for k, v in enumerate(ordered) if k % 8 == 0]
    train = [v for k, v in enumerate(ordered) if k % 8 != 0]
    assert s.test_names == [v["name"] for v in test]
    assert s.train_names == [v["name"] for v in train]
    for cams, imgs, vs in ((s.train_cameras, s.train_images, train), (s.test_cameras, s.test_images, test)):
        for cam, img, v in zip(cams, imgs, vs):
            assert (cam.width, cam.height) == (48, 32)
            assert (cam.tile_count_x, cam.tile_count_y) == (3, 2)
            assert cam.near_depth == pytest.approx(0.2)
            assert cam.far_depth == np.finfo(np.float32).max
            # downscale 1: scale 1, half-pixel shift only
            assert np.allclose([cam.fx, cam.fy, cam.cx, cam.cy], [40.0, 42.0, 23.0, 14.75])
            R = np.array(cam.R_c_w[:]).reshape(3, 3)
            assert np.allclose(R, cw.quaternion_to_matrix(v["qvec"]), atol=1e-6)
            assert np.allclose(cam.t_c_w[:], v["tvec"], atol=1e-6)
            assert np.array_equal(img, v["image"])
    assert np.allclose(s.points, pts, atol=1e-6)
    assert np.allclose(s.colors, cols / 255.0, atol=1e-7)


def _area_downscale(img, k):
    h, w = img.shape[:2]
    ow, oh = max(1, int(np.floor(w / k + 0.5))), max(1, int(np.floor(h / k + 0.5)))
    out = np.zeros((oh, ow, 3), np.uint8)
    sx, sy = w / ow, h / oh
    for y in range(oh):
        y0 = int(y * sy)
        y1 = min(h, max(y0 + 1, int((y + 1) * sy)))
        for x in range(ow):
            x0 = int(x * sx)
            x1 = min(w, max(x0 + 1, int((x + 1) * sx)))
            block = img[y0:y1, x0:x1].reshape(-1, 3).astype(np.int64)
            out[y, x] = (2 * block.sum(0) + len(block)) // (2 * len(block))
    return out


@pytest.mark.parametrize("k", [2, 3])
def test_downscale_scales_intrinsics_and_images(tmp_path, k):
    rng = np.random.default_rng(5)
    views, _, _ = _scene(tmp_path, rng, count=9, width=50, height=34)
    s = gsn.ColmapScene(tmp_path, downscale=k)
    ordered = sorted(views, key=lambda v: v["name"])
    train = [v for i, v in enumerate(ordered) if i % 8 != 0]
    cam = s.train_cameras[0]
    ow, oh = int(np.floor(50 / k + 0.5)), int(np.floor(34 / k + 0.5))
    assert (cam.width, cam.height) == (ow, oh)
    sx, sy = ow / 50.0, oh / 34.0
    assert np.allclose([cam.fx, cam.fy, cam.cx, cam.cy],
                       [40.0 * sx, 42.0 * sy, 23.5 * sx - 0.5, 15.25 * sy - 0.5], atol=1e-5)
    for img, v in zip(s.train_images, train):
        assert np.array_equal(img, _area_downscale(v["image"], k))


def test_reads_ppm_named_in_images_bin(tmp_path):
    rng = np.random.default_rng(9)
    views = _random_views(rng, 3, 16, 16)
    for v in views:
        v["name"] = v["name"].replace(".jpg", ".ppm")
    cw.write_scene(str(tmp_path), 16, 16, 10.0, 10.0, 8.0, 8.0, views, rng.normal(size=(4, 3)),
                   np.zeros((4, 3)))
    s = gsn.ColmapScene(tmp_path)
    assert len(s.train_names) == 2 and len(s.test_names) == 1


def test_error_cases(tmp_path):
    rng = np.random.default_rng(11)
    pts, cols = rng.normal(size=(4, 3)), np.zeros((4, 3))
    # non-PINHOLE camera model (SIMPLE_RADIAL = 2)
    d = tmp_path / "model"
    cw.write_scene(str(d), 16, 16, 10.0, 10.0, 8.0, 8.0, _random_views(rng, 2, 16, 16), pts, cols, model=2)
    with pytest.raises(gsn.GsnError):
        gsn.ColmapScene(d)
    # image referencing an unknown camera
    d = tmp_path / "camera"
    views = _random_views(rng, 2, 16, 16)
    views[1]["camera_id"] = 7
    cw.write_scene(str(d), 16, 16, 10.0, 10.0, 8.0, 8.0, views, pts, cols)
    with pytest.raises(gsn.GsnError):
        gsn.ColmapScene(d)
    # missing image file
    d = tmp_path / "missing"
    views = _random_views(rng, 2, 16, 16)
    views[0]["image"] = None
    cw.write_scene(str(d), 16, 16, 10.0, 10.0, 8.0, 8.0, views, pts, cols)
    with pytest.raises(gsn.GsnError):
        gsn.ColmapScene(d)
    # truncated images.bin
    d = tmp_path / "truncated"
    cw.write_scene(str(d), 16, 16, 10.0, 10.0, 8.0, 8.0, _random_views(rng, 2, 16, 16), pts, cols)
    path = d / "sparse" / "0" / "images.bin"
    data = path.read_bytes()
    path.write_bytes(data[:len(data) - 9])
    with pytest.raises(gsn.GsnError):
        gsn.ColmapScene(d)
    # no scene at all
    with pytest.raises(gsn.GsnError):
        gsn.ColmapScene(tmp_path / "absent")


@pytest.mark.parametrize("shape", [(1, 1), (7, 13), (300, 251)])
def test_png_writer_round_trip(tmp_path, shape):
    img = np.random.default_rng(1).integers(0, 256, size=shape + (3,), dtype=np.uint8)
    p = tmp_path / "x.png"
    assert gsn.write_png(p, img) == 0
    assert np.array_equal(cw.decode_png(p), img)


def test_ppm_writer_round_trip(tmp_path):
    img = np.random.default_rng(2).integers(0, 256, size=(5, 9, 3), dtype=np.uint8)
    p = tmp_path / "x.ppm"
    assert gsn.write_ppm(p, img) == 0
    data = p.read_bytes()
    assert data.startswith(b"P6\n9 5\n255\n")
    assert np.array_equal(np.frombuffer(data[len(b"P6\n9 5\n255\n"):], np.uint8).reshape(5, 9, 3), img)
