"""ctypes binding of libgsn_b200.so, the gs-native B200 C ABI (include/gsn.h).

Python here is only the FFI plumbing that the tests and the benchmark use to
drive the C ABI; device memory is passed as raw CUDA addresses (for example
``torch.Tensor.data_ptr()``). Loading fails loudly when the compiled library is
missing: there is no Python or CPU fallback for any stage.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgsn_b200.so")

PARAM_COUNT = 58
POSITION_INDEX, LOG_SCALE_INDEX, ROTATION_INDEX, OPACITY_INDEX, SH_INDEX = 0, 3, 6, 9, 10
TILE = 16

c_float_p = ctypes.POINTER(ctypes.c_float)


class Camera(ctypes.Structure):
    """Byte-compatible with gsn_camera / gs_native::CameraParams."""

    _fields_ = [
        ("fx", ctypes.c_float), ("fy", ctypes.c_float), ("cx", ctypes.c_float), ("cy", ctypes.c_float),
        ("R_c_w", ctypes.c_float * 9), ("t_c_w", ctypes.c_float * 3),
        ("near_depth", ctypes.c_float), ("far_depth", ctypes.c_float),
        ("width", ctypes.c_int), ("height", ctypes.c_int),
        ("pixel_offset", ctypes.c_int64),
        ("tile_count_x", ctypes.c_int), ("tile_count_y", ctypes.c_int),
        ("tile_offset", ctypes.c_int),
    ]

    @property
    def tiles(self):
        return self.tile_count_x * self.tile_count_y

    @property
    def pixels(self):
        return self.width * self.height


class RendererBuffers(ctypes.Structure):
    _fields_ = [
        ("means", ctypes.c_void_p), ("conic_opacity", ctypes.c_void_p), ("colors", ctypes.c_void_p),
        ("depths", ctypes.c_void_p), ("rects", ctypes.c_void_p), ("tile_counts", ctypes.c_void_p),
        ("radii", ctypes.c_void_p), ("tile_gaussian_ids", ctypes.c_void_p), ("tile_offsets", ctypes.c_void_p),
        ("contributors", ctypes.c_void_p), ("record_count", ctypes.c_void_p), ("overflow", ctypes.c_void_p),
        ("record_count_host", ctypes.c_int64), ("gaussian_capacity", ctypes.c_int),
        ("tile_capacity", ctypes.c_int),
    ]


_lib = None


class GsnError(RuntimeError):
    pass


def _check(status, what):
    if status != 0:
        raise GsnError(f"{what} failed with gsn status {status}")


def lib():
    """Loads libgsn_b200.so once; raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise GsnError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` (the CUDA path has no fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float
    P = ctypes.POINTER
    sig = {
        "gsn_version": ([], ctypes.c_char_p),
        "gsn_memcpy": ([vp, vp, ctypes.c_size_t], i32),
        "gsn_memcpy_async": ([vp, vp, ctypes.c_size_t, vp], i32),
        "gsn_stream_synchronize": ([vp], i32),
        "gsn_device_alloc": ([ctypes.c_size_t, P(vp)], i32),
        "gsn_device_free": ([vp], i32),
        "gsn_kernel_launch_count": ([], ctypes.c_uint64),
        "gsn_set_programmatic_launch": ([i32], i32),
        "gsn_profile_enable": ([i32], i32),
        "gsn_profile_collect": ([P(ctypes.c_double), i32], i32),
        "gsn_stage_name": ([i32], ctypes.c_char_p),
        "gsn_stage_count": ([], i32),
        "gsn_sort_pairs_workspace": ([i32, P(ctypes.c_size_t)], i32),
        "gsn_sort_pairs": ([vp, vp, vp, vp, i32, i32, i32, vp, ctypes.c_size_t, P(i32), vp], i32),
        "gsn_exclusive_scan_workspace": ([i32, P(ctypes.c_size_t)], i32),
        "gsn_exclusive_scan": ([vp, vp, vp, i32, vp, vp, ctypes.c_size_t, vp], i32),
        "gsn_renderer_create": ([P(vp)], i32),
        "gsn_renderer_destroy": ([vp], i32),
        "gsn_renderer_set_stream": ([vp, vp], i32),
        "gsn_renderer_render": ([vp, vp, i32, P(Camera), c_float_p, vp, i32], i32),
        "gsn_renderer_get_buffers": ([vp, P(RendererBuffers)], i32),
        "gsn_renderer_record_offsets": ([vp, P(vp)], i32),
        "gsn_renderer_set_record_capacity": ([vp, i64], i32),
        "gsn_renderer_set_bf16_sh": ([vp, i32], i32),
        "gsn_renderer_set_exact_culling": ([vp, i32], i32),
        "gsn_solver_set_bf16_sh": ([vp, i32], i32),
        "gsn_solver_set_tensor_core_loss": ([vp, i32], i32),
        "gsn_solver_status": ([vp, P(i32)], i32),
        "gsn_solver_create": ([P(vp)], i32),
        "gsn_solver_destroy": ([vp], i32),
        "gsn_solver_set_stream": ([vp, vp], i32),
        "gsn_solver_iterate": ([vp, P(Camera), vp, vp, vp, vp, i32, f32, i32], i32),
        "gsn_solver_reset_opacity_history": ([vp], i32),
        "gsn_solver_remap": ([vp, vp, i32], i32),
        "gsn_solver_statistics": ([vp, P(vp), P(vp)], i32),
        "gsn_solver_set_learning_rates": ([vp, f32, f32, f32, f32, f32], i32),
        "gsn_solver_set_compute_loss": ([vp, i32], i32),
        "gsn_solver_loss": ([vp, P(ctypes.c_double)], i32),
        "gsn_solver_loss_device": ([vp, P(vp)], i32),
        "gsn_solver_image_gradients": ([vp, P(Camera), vp, vp, P(vp)], i32),
        "gsn_solver_screen_gradients": ([vp, P(Camera), vp, vp, vp, i32, P(vp)], i32),
        "gsn_solver_map_gradients": ([vp, P(Camera), vp, vp, i32, i32, vp], i32),
        "gsn_solver_moments": ([vp, P(vp), P(vp), P(ctypes.c_uint64)], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def declare(name, args, res=ctypes.c_int):
    fn = getattr(lib(), name)
    fn.argtypes = args
    fn.restype = res
    return fn


def floats3(values):
    return (ctypes.c_float * 3)(*[float(v) for v in values])


class Renderer:
    """Handle over gs_native::Renderer (reference renderer.h:10-89)."""

    def __init__(self):
        h = ctypes.c_void_p()
        _check(lib().gsn_renderer_create(ctypes.byref(h)), "gsn_renderer_create")
        self.handle = h

    def close(self):
        if self.handle:
            lib().gsn_renderer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        _check(lib().gsn_renderer_set_stream(self.handle, ctypes.c_void_p(stream)), "set_stream")

    def render(self, params_ptr, count, camera, background, image_ptr, sh_degree):
        return lib().gsn_renderer_render(self.handle, ctypes.c_void_p(params_ptr), int(count), ctypes.byref(camera),
                                         floats3(background), ctypes.c_void_p(image_ptr), int(sh_degree))

    def buffers(self):
        b = RendererBuffers()
        _check(lib().gsn_renderer_get_buffers(self.handle, ctypes.byref(b)), "get_buffers")
        return b

    def record_offsets(self):
        p = ctypes.c_void_p()
        _check(lib().gsn_renderer_record_offsets(self.handle, ctypes.byref(p)), "record_offsets")
        return p.value

    def set_record_capacity(self, records):
        return lib().gsn_renderer_set_record_capacity(self.handle, int(records))

    def set_bf16_sh(self, enabled=True):
        _check(lib().gsn_renderer_set_bf16_sh(self.handle, int(bool(enabled))), "set_bf16_sh")

    def set_exact_culling(self, enabled=True):
        _check(lib().gsn_renderer_set_exact_culling(self.handle, int(bool(enabled))), "set_exact_culling")

    def set_fast_blend(self, enabled=True):
        fn = declare("gsn_renderer_set_fast_blend", [ctypes.c_void_p, ctypes.c_int])
        _check(fn(self.handle, int(bool(enabled))), "set_fast_blend")

    def set_pair_counter(self, device_ptr):
        fn = declare("gsn_renderer_set_pair_counter", [ctypes.c_void_p, ctypes.c_void_p])
        _check(fn(self.handle, ctypes.c_void_p(device_ptr or None)), "set_pair_counter")



def launch_count():
    return int(lib().gsn_kernel_launch_count())


def set_programmatic_launch(on=True):
    """Programmatic dependent launch of the training step's kernels (default on)."""
    _check(lib().gsn_set_programmatic_launch(int(bool(on))), "set_programmatic_launch")


def profile_enable(on=True):
    _check(lib().gsn_profile_enable(int(bool(on))), "profile_enable")


def profile_collect():
    """{stage name: device ms} since the previous collect."""
    n = lib().gsn_stage_count()
    ms = (ctypes.c_double * n)()
    _check(lib().gsn_profile_collect(ms, n), "profile_collect")
    return {lib().gsn_stage_name(k).decode(): ms[k] for k in range(n)}


def sort_pairs_workspace(max_count):
    b = ctypes.c_size_t()
    _check(lib().gsn_sort_pairs_workspace(int(max_count), ctypes.byref(b)), "sort_pairs_workspace")
    return b.value


def sort_pairs(keys, values, keys_alt, values_alt, count, begin_bit, end_bit, workspace, workspace_bytes, stream=0):
    """Returns (status, result_in_alt)."""
    alt = ctypes.c_int()
    st = lib().gsn_sort_pairs(ctypes.c_void_p(keys), ctypes.c_void_p(values), ctypes.c_void_p(keys_alt),
                              ctypes.c_void_p(values_alt), int(count), int(begin_bit), int(end_bit),
                              ctypes.c_void_p(workspace), ctypes.c_size_t(workspace_bytes), ctypes.byref(alt),
                              ctypes.c_void_p(stream))
    return st, alt.value


def exclusive_scan_workspace(max_count):
    b = ctypes.c_size_t()
    _check(lib().gsn_exclusive_scan_workspace(int(max_count), ctypes.byref(b)), "exclusive_scan_workspace")
    return b.value


def exclusive_scan(inp, gather, out, count, valid, workspace, workspace_bytes, stream=0):
    """Device pointers (gather and valid may be 0). Returns the status."""
    return lib().gsn_exclusive_scan(ctypes.c_void_p(inp), ctypes.c_void_p(gather), ctypes.c_void_p(out), int(count),
                                    ctypes.c_void_p(valid), ctypes.c_void_p(workspace),
                                    ctypes.c_size_t(workspace_bytes), ctypes.c_void_p(stream))


def device_alloc(nbytes):
    p = ctypes.c_void_p()
    _check(lib().gsn_device_alloc(ctypes.c_size_t(nbytes), ctypes.byref(p)), "gsn_device_alloc")
    return p.value or 0


def device_free(ptr):
    _check(lib().gsn_device_free(ctypes.c_void_p(ptr)), "gsn_device_free")


def memcpy_async(dst, src, nbytes, stream):
    _check(lib().gsn_memcpy_async(ctypes.c_void_p(dst), ctypes.c_void_p(src), ctypes.c_size_t(nbytes),
                                  ctypes.c_void_p(stream)), "gsn_memcpy_async")


def memcpy(dst, src, nbytes):
    _check(lib().gsn_memcpy(ctypes.c_void_p(dst), ctypes.c_void_p(src), ctypes.c_size_t(nbytes)), "gsn_memcpy")


class Solver:
    """Handle over gs_native::Solver (reference solver.h:11-68)."""

    def __init__(self):
        h = ctypes.c_void_p()
        _check(lib().gsn_solver_create(ctypes.byref(h)), "gsn_solver_create")
        self.handle = h

    def close(self):
        if self.handle:
            lib().gsn_solver_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        _check(lib().gsn_solver_set_stream(self.handle, ctypes.c_void_p(stream)), "set_stream")

    def iterate(self, camera, renderer, image_ptr, target_ptr, params_ptr, count, position_lr, sh_degree):
        return lib().gsn_solver_iterate(self.handle, ctypes.byref(camera), renderer.handle, ctypes.c_void_p(image_ptr),
                                        ctypes.c_void_p(target_ptr), ctypes.c_void_p(params_ptr), int(count),
                                        float(position_lr), int(sh_degree))

    def reset_opacity_history(self):
        return lib().gsn_solver_reset_opacity_history(self.handle)

    def remap(self, parents_ptr, count):
        return lib().gsn_solver_remap(self.handle, ctypes.c_void_p(parents_ptr), int(count))

    def statistics(self):
        a, b = ctypes.c_void_p(), ctypes.c_void_p()
        _check(lib().gsn_solver_statistics(self.handle, ctypes.byref(a), ctypes.byref(b)), "statistics")
        return a.value, b.value

    def set_learning_rates(self, scale, rotation, opacity, sh_dc, sh_rest):
        _check(lib().gsn_solver_set_learning_rates(self.handle, scale, rotation, opacity, sh_dc, sh_rest), "lr")

    def set_compute_loss(self, enabled=True):
        _check(lib().gsn_solver_set_compute_loss(self.handle, int(bool(enabled))), "set_compute_loss")

    def set_bf16_sh(self, enabled=True):
        _check(lib().gsn_solver_set_bf16_sh(self.handle, int(bool(enabled))), "set_bf16_sh")

    def set_sparse_adam(self, enabled=True):
        fn = declare("gsn_solver_set_sparse_adam", [ctypes.c_void_p, ctypes.c_int])
        _check(fn(self.handle, int(bool(enabled))), "set_sparse_adam")

    def set_lazy_moment_decay(self, enabled=True):
        fn = declare("gsn_solver_set_lazy_moment_decay", [ctypes.c_void_p, ctypes.c_int])
        _check(fn(self.handle, int(bool(enabled))), "set_lazy_moment_decay")

    def set_tensor_core_loss(self, enabled=True):
        _check(lib().gsn_solver_set_tensor_core_loss(self.handle, int(bool(enabled))), "set_tensor_core_loss")

    def status(self):
        out = ctypes.c_int()
        _check(lib().gsn_solver_status(self.handle, ctypes.byref(out)), "status")
        return out.value

    def loss(self):
        out = (ctypes.c_double * 4)()
        _check(lib().gsn_solver_loss(self.handle, out), "loss")
        return list(out)

    def loss_device(self):
        p = ctypes.c_void_p()
        _check(lib().gsn_solver_loss_device(self.handle, ctypes.byref(p)), "loss_device")
        return p.value

    def image_gradients(self, camera, image_ptr, target_ptr):
        p = ctypes.c_void_p()
        _check(lib().gsn_solver_image_gradients(self.handle, ctypes.byref(camera), ctypes.c_void_p(image_ptr),
                                                ctypes.c_void_p(target_ptr), ctypes.byref(p)), "image_gradients")
        return p.value

    def screen_gradients(self, camera, renderer, image_ptr, params_ptr, count):
        p = ctypes.c_void_p()
        _check(lib().gsn_solver_screen_gradients(self.handle, ctypes.byref(camera), renderer.handle,
                                                 ctypes.c_void_p(image_ptr), ctypes.c_void_p(params_ptr), int(count),
                                                 ctypes.byref(p)), "screen_gradients")
        return p.value

    def map_gradients(self, camera, renderer, params_ptr, count, sh_degree, grads_ptr):
        _check(lib().gsn_solver_map_gradients(self.handle, ctypes.byref(camera), renderer.handle,
                                              ctypes.c_void_p(params_ptr), int(count), int(sh_degree),
                                              ctypes.c_void_p(grads_ptr)), "map_gradients")

    def moments(self):
        a, b, it = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_uint64()
        _check(lib().gsn_solver_moments(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(it)), "moments")
        return a.value, b.value, it.value


class Density:
    """Handle over gs_native::DensityController (reference density_controller.h:9-83)."""

    def __init__(self):
        L = lib()
        vp, i32, f32, P = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.POINTER
        sigs = {
            "gsn_density_create": [P(vp)], "gsn_density_destroy": [vp], "gsn_density_set_stream": [vp, vp],
            "gsn_density_initialize": [vp, i32, i32], "gsn_density_accumulate": [vp, vp, vp, i32],
            "gsn_density_accumulate_observations": [vp, vp, vp, vp, i32],
            "gsn_density_reset_opacity": [vp, vp, i32, f32],
            "gsn_density_control": [vp, P(vp), P(i32), f32, f32, f32, f32, f32, ctypes.c_ulonglong, P(i32), f32],
            "gsn_density_buffers": [vp, P(vp), P(vp), P(vp)], "gsn_density_set_max_gaussians": [vp, i32],
            "gsn_density_set_bf16_sh": [vp, i32],
            "gsn_density_internals": [vp, P(vp), P(vp), P(vp), P(vp)],
        }
        for name, args in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = i32
        h = ctypes.c_void_p()
        _check(L.gsn_density_create(ctypes.byref(h)), "gsn_density_create")
        self.handle = h

    def close(self):
        if self.handle:
            lib().gsn_density_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        _check(lib().gsn_density_set_stream(self.handle, ctypes.c_void_p(stream)), "set_stream")

    def initialize(self, count, capacity):
        return lib().gsn_density_initialize(self.handle, int(count), int(capacity))

    def accumulate(self, stats_ptr, abs_ptr, count):
        return lib().gsn_density_accumulate(self.handle, ctypes.c_void_p(stats_ptr), ctypes.c_void_p(abs_ptr),
                                            int(count))

    def accumulate_observations(self, grads_ptr, radii_ptr, ids_ptr, observations):
        return lib().gsn_density_accumulate_observations(self.handle, ctypes.c_void_p(grads_ptr),
                                                         ctypes.c_void_p(radii_ptr), ctypes.c_void_p(ids_ptr),
                                                         int(observations))

    def reset_opacity(self, params_ptr, stride, max_opacity=0.01):
        return lib().gsn_density_reset_opacity(self.handle, ctypes.c_void_p(params_ptr), int(stride),
                                               float(max_opacity))

    def control(self, params_ptr, count, extent, grad_thr=0.0002, percent_dense=0.01, min_opacity=0.005,
                max_screen_size=0.0, seed=0, abs_thr=0.0):
        """Returns (status, new params ptr, new count, [added, removed])."""
        p = ctypes.c_void_p(params_ptr)
        c = ctypes.c_int(int(count))
        ch = (ctypes.c_int * 2)()
        st = lib().gsn_density_control(self.handle, ctypes.byref(p), ctypes.byref(c), float(extent), float(grad_thr),
                                       float(percent_dense), float(min_opacity), float(max_screen_size),
                                       ctypes.c_ulonglong(seed), ch, float(abs_thr))
        return st, (p.value or 0), c.value, [ch[0], ch[1]]

    def buffers(self):
        a, b, c = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _check(lib().gsn_density_buffers(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "buffers")
        return a.value, b.value, c.value

    def set_max_gaussians(self, n):
        _check(lib().gsn_density_set_max_gaussians(self.handle, int(n)), "set_max_gaussians")

    def set_bf16_sh(self, enabled=True):
        _check(lib().gsn_density_set_bf16_sh(self.handle, int(bool(enabled))), "set_bf16_sh")

    def internals(self):
        ps = [ctypes.c_void_p() for _ in range(4)]
        _check(lib().gsn_density_internals(self.handle, *[ctypes.byref(p) for p in ps]), "internals")
        return [p.value for p in ps]


def knn3_host(points, neighbors=False):
    """points: (n, 3) float32 host array -> (mean_dist2[n], neighbors[n, 3] or None)."""
    import numpy as np
    L = lib()
    fn = L.gsn_knn3_host
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    pts = np.ascontiguousarray(points, dtype=np.float32)
    n = pts.shape[0]
    d = np.zeros(n, dtype=np.float32)
    nb = np.zeros((n, 3), dtype=np.int32) if neighbors else None
    _check(fn(ctypes.c_void_p(pts.ctypes.data), n, ctypes.c_void_p(d.ctypes.data),
              ctypes.c_void_p(nb.ctypes.data) if nb is not None else None), "gsn_knn3_host")
    return d, nb


class TrainingOptions(ctypes.Structure):
    """gsn_training_options (include/gsn.h)."""

    _fields_ = [
        ("sh_degree_interval", ctypes.c_int), ("max_sh_degree", ctypes.c_int),
        ("position_lr_init", ctypes.c_float), ("position_lr_final", ctypes.c_float),
        ("position_lr_steps", ctypes.c_int),
        ("lr_scale", ctypes.c_float), ("lr_rotation", ctypes.c_float), ("lr_opacity", ctypes.c_float),
        ("lr_sh_dc", ctypes.c_float), ("lr_sh_rest", ctypes.c_float),
        ("densify_from", ctypes.c_int), ("densify_until", ctypes.c_int), ("densify_interval", ctypes.c_int),
        ("gradient_threshold", ctypes.c_float), ("absolute_gradient_threshold", ctypes.c_float),
        ("percent_dense", ctypes.c_float), ("min_opacity", ctypes.c_float), ("prune_large_after", ctypes.c_int),
        ("opacity_cap_interval", ctypes.c_int), ("opacity_cap", ctypes.c_float),
        ("opacity_reset_interval", ctypes.c_int), ("opacity_reset", ctypes.c_float),
        ("background", ctypes.c_float * 3), ("max_gaussians", ctypes.c_int),
        ("density_seed", ctypes.c_ulonglong), ("initial_opacity", ctypes.c_float),
        ("precision", ctypes.c_int), ("graph", ctypes.c_int),
        ("learned_density", ctypes.c_int), ("learned_confidence", ctypes.c_float), ("log_density", ctypes.c_int),
        ("exact_culling", ctypes.c_int), ("sparse_adam", ctypes.c_int), ("spatial_order", ctypes.c_int),
        ("fast_blend", ctypes.c_int), ("fp32_ssim", ctypes.c_int),
    ]

    @classmethod
    def defaults(cls, **overrides):
        o = cls()
        fn = lib().gsn_training_options_default
        fn.argtypes = [ctypes.POINTER(cls)]
        fn.restype = ctypes.c_int
        _check(fn(ctypes.byref(o)), "gsn_training_options_default")
        for k, v in overrides.items():
            if k == "background":
                for c in range(3):
                    o.background[c] = float(v[c])
            else:
                setattr(o, k, v)
        return o


class Trainer:
    """Handle over gs_native::GaussianSplatting (reference gaussian_splatting.h:14-53)."""

    def __init__(self):
        L = lib()
        vp, i32, P = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER
        sigs = {
            "gsn_trainer_create": [P(vp)], "gsn_trainer_destroy": [vp], "gsn_trainer_set_stream": [vp, vp],
            "gsn_trainer_initialize": [vp, P(Camera), P(vp), i32, vp, vp, i32, P(TrainingOptions)],
            "gsn_trainer_train": [vp, i32], "gsn_trainer_render": [vp, P(Camera), vp],
            "gsn_trainer_evaluate": [vp, P(Camera), P(vp), i32, P(ctypes.c_double), P(ctypes.c_double)],
            "gsn_trainer_save": [vp, ctypes.c_char_p], "gsn_trainer_load": [vp, ctypes.c_char_p],
            "gsn_trainer_state": [vp, P(vp), P(i32), P(i32), P(i32), P(ctypes.c_float)],
            "gsn_trainer_set_density_mlp": [vp, P(ctypes.c_float)],
            "gsn_trainer_save_checkpoint": [vp, ctypes.c_char_p], "gsn_trainer_load_checkpoint": [vp, ctypes.c_char_p],
            "gsn_trainer_evaluate_metrics": [vp, P(Camera), P(vp), i32, P(ctypes.c_double), P(ctypes.c_double),
                                             P(ctypes.c_double), P(ctypes.c_double)],
            "gsn_trainer_density_log": [vp, P(vp), P(vp), P(vp), P(i32), P(i32), P(i32), P(i32)],
        }
        for name, args in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = i32
        h = ctypes.c_void_p()
        _check(L.gsn_trainer_create(ctypes.byref(h)), "gsn_trainer_create")
        self.handle = h

    def close(self):
        if self.handle:
            lib().gsn_trainer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        _check(lib().gsn_trainer_set_stream(self.handle, ctypes.c_void_p(stream)), "set_stream")

    @staticmethod
    def _views(cameras, images):
        import numpy as np
        cams = (Camera * len(cameras))(*cameras)
        keep = [np.ascontiguousarray(im, dtype=np.uint8) for im in images]
        ptrs = (ctypes.c_void_p * len(keep))(*[im.ctypes.data for im in keep])
        return cams, ptrs, keep

    def initialize(self, cameras, images, points, colors, options=None):
        import numpy as np
        cams, ptrs, keep = self._views(cameras, images)
        pts = np.ascontiguousarray(points, dtype=np.float32)
        col = np.ascontiguousarray(colors, dtype=np.float32)
        opt = ctypes.byref(options) if options is not None else None
        return lib().gsn_trainer_initialize(self.handle, cams, ptrs, len(cameras), ctypes.c_void_p(pts.ctypes.data),
                                            ctypes.c_void_p(col.ctypes.data), pts.shape[0], opt)

    def train(self, iterations):
        return lib().gsn_trainer_train(self.handle, int(iterations))

    def set_lazy_moment_decay(self, enabled=True):
        fn = declare("gsn_trainer_set_lazy_moment_decay", [ctypes.c_void_p, ctypes.c_int])
        _check(fn(self.handle, int(bool(enabled))), "set_lazy_moment_decay")

    def render(self, camera, image_ptr):
        return lib().gsn_trainer_render(self.handle, ctypes.byref(camera), ctypes.c_void_p(image_ptr))

    def evaluate(self, cameras, images):
        cams, ptrs, keep = self._views(cameras, images)
        psnr, loss = ctypes.c_double(), ctypes.c_double()
        _check(lib().gsn_trainer_evaluate(self.handle, cams, ptrs, len(cameras), ctypes.byref(psnr),
                                          ctypes.byref(loss)), "evaluate")
        return psnr.value, loss.value

    def evaluate_metrics(self, cameras, images):
        """Mean FP64 PSNR, SSIM and L1 of the clamped renders and the mean
        training loss over the views."""
        cams, ptrs, keep = self._views(cameras, images)
        out = [ctypes.c_double() for _ in range(4)]
        _check(lib().gsn_trainer_evaluate_metrics(self.handle, cams, ptrs, len(cameras), *[ctypes.byref(o) for o in out]),
               "evaluate_metrics")
        return dict(psnr=out[0].value, ssim=out[1].value, l1=out[2].value, loss=out[3].value)

    def save(self, path):
        return lib().gsn_trainer_save(self.handle, str(path).encode())

    def load(self, path):
        return lib().gsn_trainer_load(self.handle, str(path).encode())

    def state(self):
        p, n, c, s, e = ctypes.c_void_p(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        _check(lib().gsn_trainer_state(self.handle, ctypes.byref(p), ctypes.byref(n), ctypes.byref(c),
                                       ctypes.byref(s), ctypes.byref(e)), "state")
        return dict(params=p.value or 0, count=n.value, completed=c.value, sh_degree=s.value, extent=e.value)


def ply_write(path, params):
    import numpy as np
    L = lib()
    L.gsn_ply_write.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int]
    L.gsn_ply_write.restype = ctypes.c_int
    p = np.ascontiguousarray(params, dtype=np.float32)
    return L.gsn_ply_write(str(path).encode(), ctypes.c_void_p(p.ctypes.data), p.shape[1])


def ply_read(path):
    """Returns (status, (58, n) float32 array or None)."""
    import numpy as np
    L = lib()
    L.gsn_ply_read_count.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
    L.gsn_ply_read_count.restype = ctypes.c_int
    L.gsn_ply_read.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int]
    L.gsn_ply_read.restype = ctypes.c_int
    n = ctypes.c_int()
    st = L.gsn_ply_read_count(str(path).encode(), ctypes.byref(n))
    if st != 0:
        return st, None
    out = np.zeros((58, n.value), dtype=np.float32)
    st = L.gsn_ply_read(str(path).encode(), ctypes.c_void_p(out.ctypes.data), n.value)
    return st, out


class Graph:
    """Batched form: one CUDA graph per training iteration, replayed from a
    device schedule (gs-native extension, include/gsn.h "batched form")."""

    def __init__(self):
        L = lib()
        vp, i32, i64, P = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.POINTER
        sigs = {
            "gsn_graph_create": [P(vp)], "gsn_graph_destroy": [vp],
            "gsn_graph_capture": [vp, vp, vp, vp, i32, P(Camera), i32, vp, ctypes.c_size_t, c_float_p, vp, i32,
                                  i64, vp],
            "gsn_graph_run": [vp, P(i32), P(ctypes.c_float), i32], "gsn_graph_check": [vp],
            "gsn_graph_launches_per_step": [vp, P(i32)],
        }
        for name, args in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = i32
        h = ctypes.c_void_p()
        _check(L.gsn_graph_create(ctypes.byref(h)), "gsn_graph_create")
        self.handle = h
        self._keep = []

    def close(self):
        if self.handle:
            lib().gsn_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def capture(self, renderer, solver, params_ptr, count, cameras, targets_ptr, target_stride, background,
                image_ptr, sh_degree, record_capacity, stream=0):
        cams = (Camera * len(cameras))(*cameras)
        bg = floats3(background)
        self._keep = [cams, bg, renderer, solver]
        _check(lib().gsn_graph_capture(self.handle, renderer.handle, solver.handle, ctypes.c_void_p(params_ptr),
                                       int(count), cams, len(cameras), ctypes.c_void_p(targets_ptr),
                                       int(target_stride), bg, ctypes.c_void_p(image_ptr), int(sh_degree),
                                       int(record_capacity), ctypes.c_void_p(stream)), "gsn_graph_capture")

    def run(self, views, position_lrs):
        n = len(views)
        assert len(position_lrs) == n
        v = (ctypes.c_int * n)(*[int(x) for x in views])
        lr = (ctypes.c_float * n)(*[float(x) for x in position_lrs])
        _check(lib().gsn_graph_run(self.handle, v, lr, n), "gsn_graph_run")

    def check(self):
        """0, or the gsn status (GSN_ERR_CAPACITY = -4 on a record overflow)."""
        return lib().gsn_graph_check(self.handle)

    def launches_per_step(self):
        out = ctypes.c_int()
        _check(lib().gsn_graph_launches_per_step(self.handle, ctypes.byref(out)), "launches_per_step")
        return out.value


def to_precision_layout(params, torch):
    """58 x N fp32 parameter block (numpy or torch) -> the precision-form device
    block: 10 fp32 geometry rows, then the 48 SH coefficients in bf16 as 24 rows
    of pairs (34 float rows; coefficient 2r in the low half of word r * N + i
    of the SH block, 2r + 1 in its high half)."""
    p = torch.as_tensor(params).cuda().float()
    n = p.shape[1]
    block = torch.empty(34 * n, dtype=torch.float32, device="cuda")
    block[:10 * n] = p[:10].reshape(-1)
    pairs = p[10:].reshape(24, 2, n).transpose(1, 2).to(torch.bfloat16)
    block[10 * n:].view(torch.bfloat16)[:] = pairs.reshape(-1)
    return block


def from_precision_layout(block, n, torch):
    """Inverse of to_precision_layout: a 58 x N fp32 tensor (SH widened)."""
    out = torch.empty((58, n), dtype=torch.float32, device=block.device)
    out[:10] = block[:10 * n].reshape(10, n)
    out[10:] = block[10 * n:34 * n].view(torch.bfloat16).reshape(24, n, 2).transpose(1, 2).reshape(48, n).float()
    return out


def _trainer_set_density_mlp(self, weights):
    import numpy as np
    w = np.ascontiguousarray(weights, dtype=np.float32)
    assert w.size == MLP_PARAMS
    _check(lib().gsn_trainer_set_density_mlp(self.handle, w.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
           "set_density_mlp")


def _trainer_density_log(self):
    f, d, p = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    b, a, s, it = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib().gsn_trainer_density_log(self.handle, ctypes.byref(f), ctypes.byref(d), ctypes.byref(p),
                                         ctypes.byref(b), ctypes.byref(a), ctypes.byref(s), ctypes.byref(it)),
           "density_log")
    return dict(features=f.value, decisions=d.value, parents=p.value, before=b.value, after=a.value, steps=s.value,
                iteration=it.value)


Trainer.set_density_mlp = _trainer_set_density_mlp
Trainer.save_checkpoint = lambda self, path: lib().gsn_trainer_save_checkpoint(self.handle, str(path).encode())
Trainer.load_checkpoint = lambda self, path: lib().gsn_trainer_load_checkpoint(self.handle, str(path).encode())
Trainer.density_log = _trainer_density_log

MLP_PARAMS = 5508


class Mlp:
    """Learned density policy network (include/gsn.h "learned density MLP")."""

    def __init__(self, seed=0):
        L = lib()
        vp, i32, P = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER
        sigs = {
            "gsn_mlp_create": [P(vp)], "gsn_mlp_destroy": [vp], "gsn_mlp_initialize": [vp, ctypes.c_ulonglong],
            "gsn_mlp_set_weights": [vp, P(ctypes.c_float)], "gsn_mlp_get_weights": [vp, P(ctypes.c_float)],
            "gsn_mlp_gradients": [vp, vp, vp, vp, i32, P(ctypes.c_float), P(ctypes.c_double)],
            "gsn_mlp_train": [vp, vp, vp, vp, i32, i32, ctypes.c_float, P(ctypes.c_double)],
            "gsn_mlp_infer": [vp, vp, i32, ctypes.c_float, vp, vp],
        }
        for name, args in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = i32
        h = ctypes.c_void_p()
        _check(L.gsn_mlp_create(ctypes.byref(h)), "gsn_mlp_create")
        self.handle = h
        _check(L.gsn_mlp_initialize(h, seed), "gsn_mlp_initialize")

    def close(self):
        if self.handle:
            lib().gsn_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def weights(self):
        import numpy as np
        w = np.zeros(MLP_PARAMS, np.float32)
        _check(lib().gsn_mlp_get_weights(self.handle, w.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
               "get_weights")
        return w

    def set_weights(self, w):
        import numpy as np
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(lib().gsn_mlp_set_weights(self.handle, w.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
               "set_weights")

    def gradients(self, features_ptr, labels_ptr, weights_ptr, n):
        import numpy as np
        g = np.zeros(MLP_PARAMS, np.float32)
        loss = ctypes.c_double()
        _check(lib().gsn_mlp_gradients(self.handle, ctypes.c_void_p(features_ptr), ctypes.c_void_p(labels_ptr),
                                       ctypes.c_void_p(weights_ptr), int(n),
                                       g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(loss)),
               "gradients")
        return g, loss.value

    def train(self, features_ptr, labels_ptr, weights_ptr, n, steps, lr):
        loss = ctypes.c_double()
        _check(lib().gsn_mlp_train(self.handle, ctypes.c_void_p(features_ptr), ctypes.c_void_p(labels_ptr),
                                   ctypes.c_void_p(weights_ptr), int(n), int(steps), float(lr), ctypes.byref(loss)),
               "train")
        return loss.value

    def infer(self, features_ptr, n, confidence, actions_ptr, probs_ptr=0):
        _check(lib().gsn_mlp_infer(self.handle, ctypes.c_void_p(features_ptr), int(n), float(confidence),
                                   ctypes.c_void_p(actions_ptr), ctypes.c_void_p(probs_ptr or None)), "infer")


class MultiView:
    """Multi-view renderer with one persistent blend launch and its autotuner
    (include/gsn.h "multi-view renderer")."""

    def __init__(self):
        L = lib()
        vp, i32, P = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER
        sigs = {
            "gsn_multiview_create": [P(vp)], "gsn_multiview_destroy": [vp], "gsn_multiview_set_stream": [vp, vp],
            "gsn_multiview_set_config": [vp, i32, i32, i32, i32],
            "gsn_multiview_get_config": [vp, P(i32), P(i32), P(i32), P(i32)],
            "gsn_multiview_render": [vp, vp, i32, P(Camera), i32, P(vp), c_float_p, i32],
            "gsn_multiview_autotune": [vp, vp, i32, P(Camera), i32, P(vp), c_float_p, i32, i32, c_float_p, i32,
                                       P(i32)],
        }
        for name, args in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = i32
        h = ctypes.c_void_p()
        _check(L.gsn_multiview_create(ctypes.byref(h)), "gsn_multiview_create")
        self.handle = h

    def close(self):
        if self.handle:
            lib().gsn_multiview_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        _check(lib().gsn_multiview_set_stream(self.handle, ctypes.c_void_p(stream)), "set_stream")

    def set_config(self, tile_w=16, tile_h=16, threads=64, key_bits=32):
        _check(lib().gsn_multiview_set_config(self.handle, tile_w, tile_h, threads, key_bits), "set_config")

    def config(self):
        v = [ctypes.c_int() for _ in range(4)]
        _check(lib().gsn_multiview_get_config(self.handle, *[ctypes.byref(x) for x in v]), "get_config")
        return tuple(x.value for x in v)

    @staticmethod
    def _inputs(cameras, image_ptrs):
        cams = (Camera * len(cameras))(*cameras)
        imgs = (ctypes.c_void_p * len(image_ptrs))(*[ctypes.c_void_p(p) for p in image_ptrs])
        return cams, imgs

    def render(self, params_ptr, count, cameras, image_ptrs, background, sh_degree):
        cams, imgs = self._inputs(cameras, image_ptrs)
        _check(lib().gsn_multiview_render(self.handle, ctypes.c_void_p(params_ptr), int(count), cams, len(cameras),
                                          imgs, floats3(background), int(sh_degree)), "multiview_render")

    def autotune(self, params_ptr, count, cameras, image_ptrs, background, sh_degree, repeats=2):
        cams, imgs = self._inputs(cameras, image_ptrs)
        res = (ctypes.c_float * (5 * 64))()
        n = ctypes.c_int()
        _check(lib().gsn_multiview_autotune(self.handle, ctypes.c_void_p(params_ptr), int(count), cams, len(cameras),
                                            imgs, floats3(background), int(sh_degree), int(repeats), res, 64,
                                            ctypes.byref(n)), "multiview_autotune")
        return [dict(tile_w=int(res[5 * k]), tile_h=int(res[5 * k + 1]), threads=int(res[5 * k + 2]),
                     key_bits=int(res[5 * k + 3]), ms=float(res[5 * k + 4])) for k in range(min(n.value, 64))]


class ColmapScene:
    """COLMAP scene read without OpenCV (include/gsn.h "COLMAP scene"): train /
    test cameras (Camera), host u8 HWC images (numpy views copied out), image
    names and the sparse point cloud."""

    def __init__(self, scene_dir, downscale=1):
        import numpy as np
        vp, i32, P = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER
        read = declare("gsn_scene_read_colmap", [ctypes.c_char_p, i32, P(vp)])
        counts = declare("gsn_scene_counts", [vp, P(i32), P(i32), P(i32)])
        view = declare("gsn_scene_view", [vp, i32, i32, P(Camera), P(ctypes.POINTER(ctypes.c_uint8)),
                                          P(ctypes.c_char_p)])
        points = declare("gsn_scene_points", [vp, P(c_float_p), P(c_float_p)])
        destroy = declare("gsn_scene_destroy", [vp])
        handle = vp()
        _check(read(str(scene_dir).encode(), int(downscale), ctypes.byref(handle)), "scene_read_colmap")
        try:
            n = [ctypes.c_int() for _ in range(3)]
            _check(counts(handle, *[ctypes.byref(x) for x in n]), "scene_counts")
            self.train_cameras, self.test_cameras = [], []
            self.train_images, self.test_images = [], []
            self.train_names, self.test_names = [], []
            for split, (cams, imgs, names) in enumerate(
                    [(self.train_cameras, self.train_images, self.train_names),
                     (self.test_cameras, self.test_images, self.test_names)]):
                for k in range(n[split].value):
                    cam, img, name = Camera(), ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_char_p()
                    _check(view(handle, split, k, ctypes.byref(cam), ctypes.byref(img), ctypes.byref(name)),
                           "scene_view")
                    cams.append(cam)
                    imgs.append(np.ctypeslib.as_array(img, shape=(cam.height, cam.width, 3)).copy())
                    names.append(name.value.decode())
            pos, col = c_float_p(), c_float_p()
            _check(points(handle, ctypes.byref(pos), ctypes.byref(col)), "scene_points")
            m = n[2].value
            self.points = np.ctypeslib.as_array(pos, shape=(m, 3)).copy() if m else np.zeros((0, 3), np.float32)
            self.colors = np.ctypeslib.as_array(col, shape=(m, 3)).copy() if m else np.zeros((0, 3), np.float32)
        finally:
            destroy(handle)


def write_png(path, rgb):
    """8-bit RGB PNG (HWC uint8 array)."""
    import numpy as np
    a = np.ascontiguousarray(rgb, dtype=np.uint8)
    fn = declare("gsn_image_write_png", [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int])
    return fn(str(path).encode(), ctypes.c_void_p(a.ctypes.data), a.shape[1], a.shape[0])


def write_ppm(path, rgb):
    """Binary PPM (P6) of an HWC uint8 array."""
    import numpy as np
    a = np.ascontiguousarray(rgb, dtype=np.uint8)
    fn = declare("gsn_image_write_ppm", [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int])
    return fn(str(path).encode(), ctypes.c_void_p(a.ctypes.data), a.shape[1], a.shape[0])


def eval_metrics(image_ptr, target_ptr, width, height, stream=0):
    """FP64 held-out-view metrics of one device fp32 HWC render against a device
    u8 HWC target: dict(psnr, ssim, l1, mse) with the render clamped to [0, 1]."""
    fn = declare("gsn_eval_metrics", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_double), ctypes.c_void_p])
    out = (ctypes.c_double * 4)()
    _check(fn(ctypes.c_void_p(image_ptr), ctypes.c_void_p(target_ptr), int(width), int(height), out,
              ctypes.c_void_p(stream)), "eval_metrics")
    return dict(psnr=out[0], ssim=out[1], l1=out[2], mse=out[3])


def spatial_permutation(params_ptr, count, perm_ptr, stream=0):
    """Morton-order permutation of a device parameter block into perm (device uint32[count])."""
    fn = declare("gsn_spatial_permutation", [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p])
    _check(fn(ctypes.c_void_p(params_ptr), int(count), ctypes.c_void_p(perm_ptr), ctypes.c_void_p(stream)),
           "spatial_permutation")


def gather_gaussians(src_ptr, dst_ptr, perm_ptr, count, bf16_sh=False, stream=0):
    """dst[r][i] = src[r][perm[i]] over a device parameter / moment block."""
    fn = declare("gsn_gather_gaussians", [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_void_p])
    _check(fn(ctypes.c_void_p(src_ptr), ctypes.c_void_p(dst_ptr), ctypes.c_void_p(perm_ptr), int(count),
              int(bool(bf16_sh)), ctypes.c_void_p(stream)), "gather_gaussians")

