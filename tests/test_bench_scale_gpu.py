"""GPU parity at the benchmarked configuration: the bench's 1.2M-Gaussian model
(seed 8, means N(0, 3^2)) seen from ring view 0 at 1600x1064 (fx = fy = 1400,
6,700 tiles, ~12.1M records: 13 tile bits, multi-chunk sorts, int64 offsets),
target rendered from the hidden 1.5M-Gaussian model (seed 7).

The plain form against the reference's own CUDA build on identical device
inputs (renderer.cu:359-372 and 446-590; solver.cu:26-168, 325-623, 702-720):
projection outputs, per-tile lists and offsets bit-exact, image within 1e-5,
image gradient to float rounding, screen-space and mapped gradients within
1e-4 relative (the float-atomic summation order of the backward, with a floor
scaled by each row's largest value), one Adam step within a thousandth of the
step. Then the chosen form (bf16 SH storage, exact culling, fast blend
arithmetic, fp32 SSIM gradient) against the plain form on the same
bf16-rounded inputs, with the deviation bounds stated in each assertion."""
import ctypes

import numpy as np
import pytest

import gsn
import oracle
import scenes
from helpers import (RefRenderer, dev, empty, gsn_sorted_lists, host, ref_project, ref_sorted_lists, sync,
                     torch)

pytestmark = pytest.mark.gpu

V, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
SH = 3
LR = 1e-4


def need_ref():
    if not oracle.ref_available():
        pytest.skip("reference CUDA build (oracle/_ref) not available")


@pytest.fixture(scope="module")
def case():
    """Model, camera and u8 target of the bench workload's first step."""
    t = torch()
    hidden = scenes.random_gaussians(1_500_000, 7, mean_sigma=3.0)
    model = scenes.random_gaussians(1_200_000, 8, mean_sigma=3.0)
    train, _ = scenes.training_scene_cameras()
    cam = train[0]
    hp = dev(hidden)
    img = empty((cam.height, cam.width, 3), t.float32)
    r = gsn.Renderer()
    assert r.render(hp.data_ptr(), hp.shape[1], cam, [0, 0, 0], img.data_ptr(), SH) == 0
    target = (img * 255.0).round().clamp(0, 255).to(t.uint8)
    sync()
    return model, cam, target.cpu().numpy()


def rows_close(mine, ref, rel=1e-4, floor=1e-5):
    """Per row: |a - b| <= rel * |b| + floor * max|b|."""
    scale = np.abs(ref).max(axis=-1, keepdims=True)
    return np.abs(mine - ref) <= rel * np.abs(ref) + floor * scale


class Plain:
    """One frame of the plain form: render, image gradient, screen gradients."""

    def __init__(self, params, cam, target, precision=False):
        t = torch()
        self.n = params.shape[1]
        self.cam = cam
        self.p = gsn.to_precision_layout(params, t) if precision else dev(params)
        self.target = dev(target)
        self.image = empty((cam.height, cam.width, 3), t.float32)
        self.renderer, self.solver = gsn.Renderer(), gsn.Solver()
        self.solver.set_compute_loss(True)
        if precision:
            # the chosen form's switches (the bench's spatial order only renumbers Gaussians)
            self.renderer.set_bf16_sh(True)
            self.renderer.set_exact_culling(True)
            self.renderer.set_fast_blend(True)
            self.solver.set_bf16_sh(True)
            self.solver.set_tensor_core_loss(False)  # the benched form keeps the fp32 SSIM kernel
            self.solver.set_sparse_adam(True)
        assert self.renderer.render(self.p.data_ptr(), self.n, cam, [0, 0, 0], self.image.data_ptr(), SH) == 0
        sync()

    def image_gradients(self):
        ptr = self.solver.image_gradients(self.cam, self.image.data_ptr(), self.target.data_ptr())
        sync()
        return ptr

    def screen(self):
        gptr = self.image_gradients()
        ptr = self.solver.screen_gradients(self.cam, self.renderer, self.image.data_ptr(), self.p.data_ptr(), self.n)
        sync()
        return gptr, host(ptr, np.float32, 12 * self.n).reshape(self.n, 12)


def test_plain_projection_tile_lists_and_image_match_reference_bit_for_bit(case):
    need_ref()
    params, cam, _ = case
    t = torch()
    n = params.shape[1]
    f = Plain(params, cam, np.zeros((cam.height, cam.width, 3), np.uint8))
    rimg = empty((cam.height, cam.width, 3), t.float32)
    rr = RefRenderer()
    assert rr.render(f.p.data_ptr(), n, cam, [0, 0, 0], rimg.data_ptr(), SH) == 0
    sync()
    # projection (ProjectGaussiansKernel outputs of every visible Gaussian)
    b = f.renderer.buffers()
    counts = host(b.tile_counts, np.int32, n)
    ref = ref_project(f.p.data_ptr(), n, cam, SH)
    assert np.array_equal(counts, ref["counts"])
    vis = counts > 0
    assert vis.sum() > 500_000
    mine = dict(means=host(b.means, np.float32, 2 * n).reshape(n, 2),
                conic=host(b.conic_opacity, np.float32, 4 * n).reshape(n, 4),
                colors=host(b.colors, np.float32, 3 * n).reshape(n, 3),
                depths=host(b.depths, np.float32, n), rects=host(b.rects, np.int32, 4 * n).reshape(n, 4))
    for key, a in mine.items():
        x, y = a[vis], ref[key][vis]
        assert np.array_equal(x.view(np.uint32) if x.dtype == np.float32 else x,
                              y.view(np.uint32) if y.dtype == np.float32 else y), key
    # per-tile lists and int64 offsets of all ~12.1M records
    ids, offsets = gsn_sorted_lists(f.renderer, cam)
    r_ids, r_offsets = ref_sorted_lists(rr, cam)
    assert offsets[-1] > 10_000_000
    assert np.array_equal(offsets, r_offsets)
    assert np.array_equal(ids, r_ids)
    # image
    err = np.abs(f.image.cpu().numpy() - rimg.cpu().numpy()).max()
    print(f"bench-scale plain vs reference: records {offsets[-1]}, visible {vis.sum()}, max |image diff| {err:.3e}")
    assert err <= 1e-5


def test_plain_gradients_and_adam_step_match_reference(case):
    need_ref()
    params, cam, target = case
    t = torch()
    n = params.shape[1]
    f = Plain(params, cam, target)
    gptr, screen = f.screen()
    # image gradient (ComputeImageGradientsKernel, same tap order)
    mine_g = host(gptr, np.float32, cam.pixels * 3)
    rg = empty((cam.height, cam.width, 3), t.float32)
    fn = oracle.ref_fn("ref_image_gradients", [V, V, V, I, I])
    assert fn(V(f.image.data_ptr()), V(f.target.data_ptr()), V(rg.data_ptr()), cam.width, cam.height) == 0
    ref_g = rg.cpu().numpy().reshape(-1)
    assert np.abs(mine_g - ref_g).max() <= 1e-6 * np.abs(ref_g).max()
    # screen-space gradients (ComputeSplatGradientsKernel on the same lists)
    b = f.renderer.buffers()
    grads = empty((58, n), t.float32)
    absolute = empty((2, n), t.float32)
    fn = oracle.ref_fn("ref_splat_gradients", [V] * 7 + [V, V, V, I])
    assert fn(V(b.tile_gaussian_ids), V(b.tile_offsets), V(b.means), V(b.conic_opacity), V(b.colors),
              V(f.image.data_ptr()), V(gptr), ctypes.byref(cam), V(grads.data_ptr()), V(absolute.data_ptr()),
              n) == 0
    ref9, ref_abs = grads.cpu().numpy()[:9], absolute.cpu().numpy()
    ok9 = rows_close(screen[:, :9].T, ref9)
    ok_abs = rows_close(screen[:, 9:11].T, ref_abs)
    rel_l2 = np.linalg.norm(screen[:, :9].T - ref9, axis=1) / np.linalg.norm(ref9, axis=1)
    print(f"bench-scale screen gradients: share within 1e-4 rel + 1e-5 max-floor {ok9.mean():.7f}, "
          f"abs rows {ok_abs.mean():.7f}, per-row relative L2 max {rel_l2.max():.2e}")
    # float-atomic order: every row's relative L2 error within 1e-4, and all but
    # a few in a million elements within the element bound
    assert rel_l2.max() <= 1e-4
    assert ok9.mean() >= 1 - 1e-5 and ok_abs.mean() >= 1 - 1e-5
    # chain rule on the same screen-space input (MapGaussianGradientsKernel<3>)
    mapped = empty((58, n), t.float32)
    f.solver.map_gradients(cam, f.renderer, f.p.data_ptr(), n, SH, mapped.data_ptr())
    sync()
    ref58 = np.zeros((58, n), dtype=np.float32)
    ref58[:9] = screen[:, :9].T
    rg58 = dev(ref58)
    fn = oracle.ref_fn("ref_map_gradients", [V, V, V, I, I])
    assert fn(V(f.p.data_ptr()), ctypes.byref(cam), V(rg58.data_ptr()), n, SH) == 0
    a, r = mapped.cpu().numpy(), rg58.cpu().numpy()
    okm = rows_close(a, r, rel=1e-4, floor=1e-6)
    print(f"bench-scale mapped gradients: share within 1e-4 rel {okm.mean():.7f}, bit-identical {np.mean(a == r):.4f}")
    assert okm.all()
    # one full Iterate (loss gradient, backward, statistics, chain rule, Adam)
    step = Plain(params, cam, target)
    assert step.solver.iterate(cam, step.renderer, step.image.data_ptr(), step.target.data_ptr(),
                               step.p.data_ptr(), n, LR, SH) == 0
    sync()
    mine_p = step.p.cpu().numpy()
    rp = dev(params)
    rimg = empty((cam.height, cam.width, 3), t.float32)
    rr = RefRenderer()
    assert rr.render(rp.data_ptr(), n, cam, [0, 0, 0], rimg.data_ptr(), SH) == 0
    h = V()
    oracle.ref_fn("ref_solver_create", [ctypes.POINTER(V)])(ctypes.byref(h))
    it = oracle.ref_fn("ref_solver_iterate", [V, V, V, V, V, V, I, F, I])
    assert it(h, ctypes.byref(cam), rr.h, V(rimg.data_ptr()), V(step.target.data_ptr()), V(rp.data_ptr()), n, LR,
              SH) == 0
    ref_p = rp.cpu().numpy()
    oracle.ref_fn("ref_solver_destroy", [V])(h)
    # Adam's first step moves a parameter with a nonzero gradient by about its
    # learning rate whatever the gradient's size: parameters agree to a
    # thousandth of their step except where a gradient at rounding level
    # changes sign between the two summation orders
    diff = np.abs(mine_p - ref_p)
    moved = np.abs(ref_p - params)
    within = diff <= 1e-6 + 1e-3 * moved
    print(f"bench-scale Adam step: share within 1e-3 of the step {within.mean():.7f}")
    assert within.mean() > 0.999
    assert np.isfinite(mine_p).all()


def test_chosen_form_deviation_from_plain_at_bench_scale(case):
    """The chosen form's render and backward arithmetic (exact culling, the
    fast power / exp2 / reciprocal, 24-bit depth keys, bf16 SH storage, the
    fp32 SSIM gradient) against the plain form on the same inputs (SH already
    rounded to bf16, so storage rounding is not counted)."""
    params, cam, target = case
    t = torch()
    rounded = params.copy()
    rounded[10:] = t.from_numpy(params[10:]).to(t.bfloat16).float().numpy()
    plain = Plain(rounded, cam, target)
    chosen = Plain(rounded, cam, target, precision=True)
    img_p, img_c = plain.image.cpu().numpy(), chosen.image.cpu().numpy()
    d = np.abs(img_c - img_p)
    _, sp = plain.screen()
    _, sc = chosen.screen()
    loss_p, loss_c = plain.solver.loss()[0], chosen.solver.loss()[0]
    scale = np.abs(sp[:, :11]).max(axis=0, keepdims=True)
    bad = np.abs(sc[:, :11] - sp[:, :11]) > 1e-3 * np.abs(sp[:, :11]) + 1e-4 * scale
    rel_l2 = np.linalg.norm(sc[:, :11] - sp[:, :11], axis=0) / np.linalg.norm(sp[:, :11], axis=0)
    print(f"bench-scale chosen vs plain: image max {d.max():.3e} mean {d.mean():.3e} share > 1e-4 "
          f"{np.mean(d > 1e-4):.2e}; loss rel {abs(loss_c - loss_p) / loss_p:.2e}; screen gradients: "
          f"Gaussians outside 1e-3 rel + 1e-4 max-floor {bad.any(axis=1).mean():.2e}, per-column relative L2 "
          f"max {rel_l2.max():.2e}")
    # near-equal depths (2^-16 relative) may swap blend order on the 24-bit
    # keys, moving a few pixels by up to ~1e-2; everything else is ulp-level
    assert d.mean() < 1e-5 and np.mean(d > 1e-4) < 1e-3 and d.max() < 5e-2
    assert abs(loss_c - loss_p) <= 1e-5 * loss_p
    assert bad.any(axis=1).mean() < 5e-3
    assert rel_l2.max() < 1e-2
