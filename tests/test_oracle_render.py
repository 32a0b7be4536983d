"""CPU checks of the oracle's forward model against the reference's own
known-answer tests (renderer_test.cu) and its integer record ordering."""
import math

import numpy as np
import pytest

import oracle
import scenes


def test_lower_colour_clamp_known_answer():
    # renderer_test.cu:72-88: centre pixel clamps the negative channel to 0 and
    # keeps 1.5 * 0.9 = 1.35 on the other.
    p = scenes.make_gaussians(1)
    p[0:3, 0] = [0, 0, 3]
    p[9, 0] = math.log(9.0)
    p[10, 0] = (-0.2 - 0.5) / scenes.SH_C0
    p[26, 0] = (1.5 - 0.5) / scenes.SH_C0
    cam = scenes.make_camera(9, 7)
    img = oracle.render_params(p, cam, [0, 0, 0], 0)
    assert img[3, 4, 0] == 0.0
    assert abs(img[3, 4, 1] - 1.35) < 2e-6


@pytest.mark.parametrize("count", [2, 0])
def test_empty_and_culled_scenes_give_background(count):
    # renderer_test.cu:31-46
    p = scenes.make_gaussians(2)
    p[2, 0] = 0.1
    p[2, 1] = 101
    p = p[:, :count]
    cam = scenes.make_camera(19, 17)
    bg = [0.2, 0.4, 0.6]
    img = oracle.render_params(p, cam, bg, 0)
    assert np.all(img == np.array(bg)[None, None, :])


def test_sort_records_orders_by_tile_depth_then_id():
    # three Gaussians on two tiles, two of them with identical depth bits
    cam = scenes.make_camera(32, 16)
    depth_bits = np.array([np.float32(2.0).view(np.uint32), np.float32(1.0).view(np.uint32),
                           np.float32(2.0).view(np.uint32)], dtype=np.uint32)
    rects = np.array([[0, 0, 2, 1], [1, 0, 2, 1], [0, 0, 1, 1]], dtype=np.int32)
    counts = np.array([2, 1, 1], dtype=np.int32)
    ids, offsets = oracle.sort_records(depth_bits, rects, counts, cam)
    assert list(offsets) == [0, 2, 4]
    assert list(ids) == [0, 2, 1, 0]


def test_sort_records_empty():
    cam = scenes.make_camera(32, 16)
    ids, offsets = oracle.sort_records(np.zeros(2, np.uint32), np.zeros((2, 4), np.int32), np.zeros(2, np.int32), cam)
    assert len(ids) == 0 and list(offsets) == [0, 0, 0]


def test_tile_lists_match_integer_ordering_on_single_step_scene():
    params, cam = scenes.single_step_scene()
    proj = oracle.project(params, cam, 3)
    vis = proj["visible"] != 0
    counts = np.where(vis, (proj["rect"][:, 2] - proj["rect"][:, 0]) * (proj["rect"][:, 3] - proj["rect"][:, 1]), 0)
    bits = proj["depth"].astype(np.float32).view(np.uint32)
    ids_int, off_int = oracle.sort_records(bits, proj["rect"], counts, cam)
    off_lists, ids_lists = oracle.tile_lists(proj, cam)
    assert np.array_equal(off_int, off_lists)
    # identical except where two depths collapse to the same float32
    same = ids_int == ids_lists
    assert same.mean() > 0.999
    for r in np.nonzero(~same)[0]:
        a, b = ids_int[r], ids_lists[r]
        assert np.float32(proj["depth"][a]) == np.float32(proj["depth"][b]) or \
            abs(proj["depth"][a] - proj["depth"][b]) < 1e-6 * proj["depth"][a]


def test_single_step_scene_is_nontrivial():
    params, cam = scenes.single_step_scene()
    img = oracle.render_params(params, cam, [1, 1, 1], 3)
    assert np.isfinite(img).all()
    # white background visible at the borders, Gaussians in the middle
    assert img[64, 64].min() < 0.99
    proj = oracle.project(params, cam, 3)
    assert proj["visible"].sum() > 3000
