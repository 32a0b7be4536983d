"""GPU tests of the LBVH 3-NN: the reference's KNN tests (knn_test.cu) against
the exhaustive FP64 oracle, neighbour indices against an exhaustive FP32 search
with the same distance formula, and the reference's own CUDA implementation."""
import ctypes

import numpy as np
import pytest

import gsn
import oracle

pytestmark = pytest.mark.gpu


def make_points(mode, count, rng):
    p = rng.uniform(-10, 10, (count, 3)).astype(np.float32)
    if mode == 1:
        p[:, 0] = 0
    if mode == 2:
        p[:] = 0
    if mode == 3:
        p[:, 1:] = 0
    return p


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_matches_exhaustive_search_for_boundary_and_degenerate_clouds(mode):
    # knn_test.cu:8-42
    rng = np.random.default_rng(17 + mode)
    for count in (0, 1, 2, 3, 4, 17, 256, 1025):
        pts = make_points(mode, count, rng)
        actual, _ = gsn.knn3_host(pts)
        expected, _ = oracle.knn3(pts)
        assert actual.shape == (count,)
        for i in range(count):
            if expected[i] == 0:
                assert actual[i] == 0.0, (mode, count, i)
            else:
                assert abs(actual[i] - expected[i]) <= 2e-6 * max(1.0, expected[i]), (mode, count, i)


def test_preserves_original_point_order():
    # knn_test.cu:44-53
    pts = np.array([[100, 0, 0], [0, 0, 0], [1, 0, 0], [3, 0, 0], [7, 0, 0]], dtype=np.float32)
    first, _ = gsn.knn3_host(pts)
    second, _ = gsn.knn3_host(pts[::-1].copy())
    assert np.array_equal(first, second[::-1])


def fp32_exhaustive(pts):
    """3-NN with ((dx*dx + dy*dy) + dz*dz) in float32, ties to the smaller index."""
    n = len(pts)
    out_d = np.zeros((n, 3), dtype=np.float32)
    out_i = np.full((n, 3), -1, dtype=np.int64)
    for i in range(n):
        d = pts - pts[i]
        dist = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        dist[i] = np.inf
        order = np.lexsort((np.arange(n), dist))[:3]
        out_d[i] = dist[order]
        out_i[i] = order
    return out_d, out_i


def test_neighbor_indices_equal_exhaustive_fp32_search():
    rng = np.random.default_rng(4)
    pts = rng.normal(0, 3, (4000, 3)).astype(np.float32)
    pts[100:110] = pts[200:210]  # exact duplicates -> ties
    mean, nb = gsn.knn3_host(pts, neighbors=True)
    d, idx = fp32_exhaustive(pts)
    assert np.array_equal(nb, idx)
    expected = ((d[:, 0] + d[:, 1]) + d[:, 2]) / np.float32(3.0)
    assert np.allclose(mean, expected, rtol=1e-6, atol=0)


def test_matches_reference_cuda_implementation():
    if not oracle.ref_available():
        pytest.skip("reference CUDA build not available")
    rng = np.random.default_rng(8)
    pts = rng.normal(0, 3, (100_000, 3)).astype(np.float32)
    mine, _ = gsn.knn3_host(pts)
    ref = np.zeros(len(pts), dtype=np.float32)
    fn = oracle.ref_fn("ref_knn_mean_dist2", [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p])
    assert fn(ctypes.c_void_p(pts.ctypes.data), len(pts), ctypes.c_void_p(ref.ctypes.data)) == 0
    assert np.allclose(mine, ref, rtol=2e-6, atol=0)
