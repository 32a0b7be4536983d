"""CPU tests of the Gaussian PLY writer/reader (reference io_test.cpp:72-102)."""
import os

import numpy as np

import gsn
import scenes


def test_round_trip_including_rotation(tmp_path):
    p = scenes.make_gaussians(5)
    rng = np.random.default_rng(0)
    axis = rng.normal(size=(3, 5))
    axis /= np.linalg.norm(axis, axis=0)
    p[6:9] = (axis * rng.uniform(0.1, 3.0, 5)).astype(np.float32)
    p[6:9, 0] = 0.0  # identity rotation
    path = tmp_path / "model.ply"
    assert gsn.ply_write(path, p) == 0
    st, q = gsn.ply_read(path)
    assert st == 0 and q.shape == p.shape
    rows = [r for r in range(58) if r not in (6, 7, 8)]
    assert np.array_equal(q[rows], p[rows])
    assert np.allclose(q[6:9], p[6:9], atol=2e-6)


def test_header_layout_is_the_62_float_row(tmp_path):
    p = scenes.make_gaussians(2)
    path = tmp_path / "h.ply"
    assert gsn.ply_write(path, p) == 0
    data = open(path, "rb").read()
    header, body = data.split(b"end_header\n", 1)
    assert header.count(b"property float") == 62
    assert len(body) == 2 * 62 * 4
    row = np.frombuffer(body[: 62 * 4], dtype="<f4")
    assert row[0] == p[0, 0] and row[3] == 0.0 and row[6] == p[10, 0] and row[9] == p[11, 0]


def test_truncated_and_missing_files_fail(tmp_path):
    p = scenes.make_gaussians(3)
    path = tmp_path / "t.ply"
    assert gsn.ply_write(path, p) == 0
    data = open(path, "rb").read()
    open(tmp_path / "cut.ply", "wb").write(data[:-10])
    assert gsn.ply_read(tmp_path / "cut.ply")[0] != 0
    assert gsn.ply_read(tmp_path / "missing.ply")[0] != 0
    assert not os.path.exists(tmp_path / "missing.ply")
