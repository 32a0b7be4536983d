"""Shared helpers of the parity tests: device transfers through the gsn C ABI,
and thin wrappers over the reference's own CUDA kernels (oracle/_ref)."""
import ctypes

import numpy as np

import gsn
import oracle

_torch = None


def torch():
    global _torch
    if _torch is None:
        import torch as t
        _torch = t
    return _torch


def dev(array):
    """numpy -> CUDA tensor (contiguous copy)."""
    t = torch()
    return t.from_numpy(np.ascontiguousarray(array)).cuda()


def empty(shape, dtype):
    t = torch()
    return t.zeros(shape, dtype=dtype, device="cuda")


def host(ptr, dtype, count):
    """Copies `count` elements of `dtype` at device address `ptr` into numpy."""
    out = np.zeros(int(count), dtype=dtype)
    if count:
        gsn.memcpy(out.ctypes.data, ptr, out.nbytes)
    return out


def sync():
    torch().cuda.synchronize()


# ------------------------------------------------------------------ reference
V = ctypes.c_void_p
I = ctypes.c_int
F = ctypes.c_float


class RefRenderer:
    """The reference's gs_native::Renderer (renderer.cu) through oracle/_ref."""

    def __init__(self):
        self.h = V()
        oracle.ref_fn("ref_renderer_create", [ctypes.POINTER(V)])(ctypes.byref(self.h))

    def __del__(self):
        try:
            oracle.ref_fn("ref_renderer_destroy", [V])(self.h)
        except Exception:
            pass

    def render(self, params_ptr, count, cam, background, image_ptr, sh):
        fn = oracle.ref_fn("ref_renderer_render", [V, V, I, V, V, V, I])
        bg = (ctypes.c_float * 3)(*background)
        return fn(self.h, V(params_ptr), count, ctypes.byref(cam), ctypes.cast(bg, V), V(image_ptr), sh)

    def buffers(self):
        ptrs = [V() for _ in range(6)]
        gc, tc = I(), I()
        oracle.ref_fn("ref_renderer_get", [V] + [ctypes.POINTER(V)] * 6 + [ctypes.POINTER(I)] * 2)(
            self.h, *[ctypes.byref(p) for p in ptrs], ctypes.byref(gc), ctypes.byref(tc))
        names = ["means", "conic", "colors", "tile_ids", "tile_offsets", "record_offsets"]
        out = {k: p.value for k, p in zip(names, ptrs)}
        out["gaussian_capacity"], out["tile_capacity"] = gc.value, tc.value
        return out


def ref_project(params_ptr, count, cam, sh):
    """ProjectGaussiansKernel outputs into fresh device buffers (as numpy)."""
    t = torch()
    means = empty((count, 2), t.float32)
    conic = empty((count, 4), t.float32)
    colors = empty((count, 3), t.float32)
    depths = empty((count,), t.float32)
    rects = empty((count, 4), t.int32)
    offs = empty((count + 1,), t.int32)
    fn = oracle.ref_fn("ref_project", [V, I, V, I, V, V, V, V, V, V])
    assert fn(V(params_ptr), count, ctypes.byref(cam), sh, V(means.data_ptr()), V(conic.data_ptr()),
              V(colors.data_ptr()), V(depths.data_ptr()), V(rects.data_ptr()), V(offs.data_ptr())) == 0
    return dict(means=means.cpu().numpy(), conic=conic.cpu().numpy(), colors=colors.cpu().numpy(),
                depths=depths.cpu().numpy(), rects=rects.cpu().numpy(), counts=offs.cpu().numpy()[:count])


def render_both(params, cam, background, sh):
    """Renders with gs-native and with the reference on identical device inputs."""
    t = torch()
    n = params.shape[1]
    p = dev(params)
    img = empty((cam.height, cam.width, 3), t.float32)
    r = gsn.Renderer()
    assert r.render(p.data_ptr() if n else 0, n, cam, background, img.data_ptr(), sh) == 0
    sync()
    out = dict(image=img.cpu().numpy(), renderer=r, params=p)
    if oracle.ref_available():
        rimg = empty((cam.height, cam.width, 3), t.float32)
        rr = RefRenderer()
        assert rr.render(p.data_ptr() if n else 0, n, cam, background, rimg.data_ptr(), sh) == 0
        sync()
        out["ref_image"] = rimg.cpu().numpy()
        out["ref_renderer"] = rr
    return out


def gsn_sorted_lists(renderer, cam):
    b = renderer.buffers()
    tiles = cam.tile_count_x * cam.tile_count_y
    offsets = host(b.tile_offsets, np.int64, tiles + 1)
    ids = host(b.tile_gaussian_ids, np.int32, int(offsets[-1]))
    return ids, offsets


def ref_sorted_lists(rr, cam):
    b = rr.buffers()
    tiles = cam.tile_count_x * cam.tile_count_y
    offsets = host(b["tile_offsets"], np.int64, tiles + 1)
    ids = host(b["tile_ids"], np.int32, int(offsets[-1]))
    return ids, offsets
