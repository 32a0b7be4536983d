"""ctypes bindings of the CPU oracle (liboracle.so) and of the reference's own
CUDA kernels compiled into _ref/libgsref.so.

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
benchmark's CPU-baseline leg, never by the product.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libgsref.so")
REF_CPU_PATH = os.path.join(HERE, "_ref", "libgsref_cpu.so")

_vp, _i32, _i64, _f32, _f64, _u64 = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float,
                                     ctypes.c_double, ctypes.c_uint64)


class Proj(ctypes.Structure):
    _fields_ = [("visible", ctypes.c_int), ("rect", ctypes.c_int * 4), ("depth", _f64), ("u", _f64), ("v", _f64),
                ("cov", _f64 * 3), ("conic", _f64 * 3), ("opacity", _f64), ("radius", _f64),
                ("rgb", _f64 * 3), ("rgb_raw", _f64 * 3)]


PROJ_DTYPE = np.dtype([("visible", np.int32), ("rect", np.int32, 4), ("depth", np.float64), ("u", np.float64),
                       ("v", np.float64), ("cov", np.float64, 3), ("conic", np.float64, 3),
                       ("opacity", np.float64), ("radius", np.float64), ("rgb", np.float64, 3),
                       ("rgb_raw", np.float64, 3)], align=True)
assert PROJ_DTYPE.itemsize == ctypes.sizeof(Proj)


class LR(ctypes.Structure):
    _fields_ = [("position", _f64), ("scale", _f64), ("rotation", _f64), ("opacity", _f64), ("sh_dc", _f64),
                ("sh_rest", _f64)]


REFERENCE_LR = dict(position=1e-4, scale=0.005, rotation=0.001, opacity=0.025, sh_dc=0.0025, sh_rest=0.0025 / 20)

_orc = None
_ref = None


def ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def oracle():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_PATH):
            raise RuntimeError(f"{ORACLE_PATH} missing: run `make -C {HERE}`")
        L = ctypes.CDLL(ORACLE_PATH)
        from gsn import Camera  # noqa: F401 (same struct layout)
        cp = ctypes.c_void_p
        sigs = {
            "orc_project": [cp, _i32, cp, _i32, cp],
            "orc_sort_records": [cp, cp, cp, _i32, _i32, _i32, cp, cp],
            "orc_tile_lists": [cp, _i32, cp, ctypes.POINTER(cp), ctypes.POINTER(cp)],
            "orc_free": [cp],
            "orc_render": [cp, cp, cp, cp, cp, cp, cp, cp, _i32, _i32],
            "orc_loss": [cp, cp, _i32, _i32],
            "orc_eval_metrics": [cp, cp, _i32, _i32, cp],
            "orc_loss_gradient": [cp, cp, _i32, _i32, cp, _i32, _i32],
            "orc_backward": [cp, _i32, cp, cp, cp, cp, cp, cp, cp, _i32, _i32],
            "orc_projection_statistics": [cp, _i32, cp, cp, cp, cp, cp],
            "orc_map_gradients": [cp, _i32, cp, _i32, cp, cp],
            "orc_adam": [cp, cp, cp, cp, _i32, cp, _u64],
            "orc_density_counts": [cp, _i32, cp, cp, cp, _f32, _f32, _f32, _f32, _i32, _f32, cp],
            "orc_density_apply": [cp, _i32, cp, cp, cp, cp, cp],
            "orc_knn3": [cp, _i32, cp, cp],
            "orc_set_threads": [_i32],
        }
        res = {"orc_sort_records": _i64, "orc_loss": _f64, "orc_density_apply": _i32, "orc_set_threads": _i32}
        for name, args in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res.get(name, None)
        _orc = L
    return _orc


def ref_available():
    return os.path.exists(REF_PATH)


def reference():
    """The reference's own CUDA kernels/classes (GPU only)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError(f"{REF_PATH} missing: run `make -C {HERE} ref` where the reference tree exists")
        L = ctypes.CDLL(REF_PATH)
        for name in dir(L):
            pass
        _ref = L
    return _ref


_ref_cpu = None


def ref_cpu_available():
    return os.path.exists(REF_CPU_PATH)


def ref_cpu():
    """The reference's CPU reference (test/cpu_reference.h, single-threaded as
    written), compiled unmodified against the OpenCV shim."""
    global _ref_cpu
    if _ref_cpu is None:
        if not ref_cpu_available():
            raise RuntimeError(f"{REF_CPU_PATH} missing: run `make -C {HERE} REF=<reference tree>`")
        L = ctypes.CDLL(REF_CPU_PATH)
        cp = ctypes.c_void_p
        L.ref_cpu_render.argtypes = [cp, _i32, cp, cp, _i32, cp]
        L.ref_cpu_render.restype = _i32
        L.ref_cpu_loss.argtypes = [cp, cp, _i32, _i32, ctypes.POINTER(_f64)]
        L.ref_cpu_loss.restype = _i32
        _ref_cpu = L
    return _ref_cpu


def ref_cpu_render(params, cam, background, sh_degree):
    """RenderReference (cpu_reference.h:22-116): FP64 image of the 58 x n block."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    image = np.zeros((cam.height, cam.width, 3), dtype=np.float64)
    bg = np.ascontiguousarray(background, dtype=np.float32)
    st = ref_cpu().ref_cpu_render(ptr(params), params.shape[1], cam_ref(cam), ptr(bg), int(sh_degree), ptr(image))
    if st != 0:
        raise RuntimeError("RenderReference failed")
    return image


def ref_cpu_loss(image, target):
    """ComputeLoss (cpu_reference.h:118-152): 0.8 L1 + 0.2 (1 - SSIM)."""
    image = np.ascontiguousarray(image, dtype=np.float64)
    target = np.ascontiguousarray(target, dtype=np.uint8)
    h, w = target.shape[:2]
    out = _f64()
    if ref_cpu().ref_cpu_loss(ptr(image), ptr(target), w, h, ctypes.byref(out)) != 0:
        raise RuntimeError("ComputeLoss failed")
    return out.value


def ref_fn(name, args, res=ctypes.c_int):
    fn = getattr(reference(), name)
    fn.argtypes = args
    fn.restype = res
    return fn


# ------------------------------------------------------------------ oracle API
def cam_ref(cam):
    return ctypes.byref(cam)


def project(params, cam, sh_degree):
    params = np.ascontiguousarray(params, dtype=np.float32)
    n = params.shape[1]
    out = np.zeros(n, dtype=PROJ_DTYPE)
    oracle().orc_project(ptr(params), n, cam_ref(cam), sh_degree, ptr(out))
    return out


def sort_records(depth_bits, rects, counts, cam):
    n = len(counts)
    bits = np.ascontiguousarray(depth_bits, dtype=np.uint32)
    rects = np.ascontiguousarray(rects, dtype=np.int32)
    counts = np.ascontiguousarray(counts, dtype=np.int32)
    total = int(np.sum(counts, dtype=np.int64))
    ids = np.zeros(max(total, 1), dtype=np.int32)
    offsets = np.zeros(cam.tile_count_x * cam.tile_count_y + 1, dtype=np.int64)
    r = oracle().orc_sort_records(ptr(bits), ptr(rects), ptr(counts), n, cam.tile_count_x, cam.tile_count_y,
                                  ptr(ids), ptr(offsets))
    return ids[:r], offsets


def tile_lists(proj, cam):
    off = ctypes.c_void_p()
    ids = ctypes.c_void_p()
    oracle().orc_tile_lists(ptr(proj), len(proj), cam_ref(cam), ctypes.byref(off), ctypes.byref(ids))
    tiles = cam.tile_count_x * cam.tile_count_y
    offsets = np.ctypeslib.as_array(ctypes.cast(off, ctypes.POINTER(ctypes.c_int64)), shape=(tiles + 1,)).copy()
    total = int(offsets[-1])
    if total > 0:
        idv = np.ctypeslib.as_array(ctypes.cast(ids, ctypes.POINTER(ctypes.c_int32)), shape=(total,)).copy()
    else:
        idv = np.zeros(0, dtype=np.int32)
    oracle().orc_free(off)
    oracle().orc_free(ids)
    return offsets, idv


def render(proj, cam, offsets, ids, background, tile_range=(0, 0)):
    P = cam.width * cam.height
    image = np.zeros(P * 3, dtype=np.float64)
    final_t = np.zeros(P, dtype=np.float64)
    contributors = np.zeros(P, dtype=np.int32)
    bg = np.asarray(background, dtype=np.float64)
    ids = np.ascontiguousarray(ids, dtype=np.int32) if len(ids) else np.zeros(1, dtype=np.int32)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    oracle().orc_render(ptr(proj), cam_ref(cam), ptr(offsets), ptr(ids), ptr(bg), ptr(image), ptr(final_t),
                        ptr(contributors), tile_range[0], tile_range[1])
    return image.reshape(cam.height, cam.width, 3), final_t.reshape(cam.height, cam.width), \
        contributors.reshape(cam.height, cam.width)


def render_params(params, cam, background, sh_degree):
    proj = project(params, cam, sh_degree)
    offsets, ids = tile_lists(proj, cam)
    return render(proj, cam, offsets, ids, background)[0]


def loss(image, target):
    image = np.ascontiguousarray(image, dtype=np.float64)
    target = np.ascontiguousarray(target, dtype=np.uint8)
    h, w = target.shape[:2]
    return oracle().orc_loss(ptr(image), ptr(target), w, h)


def eval_metrics(image, target):
    """(psnr_db, ssim, l1, mse) of one view with the image clamped to [0, 1]."""
    image = np.ascontiguousarray(image, dtype=np.float64)
    target = np.ascontiguousarray(target, dtype=np.uint8)
    h, w = target.shape[:2]
    out = np.zeros(4, dtype=np.float64)
    oracle().orc_eval_metrics(ptr(image), ptr(target), w, h, ptr(out))
    return tuple(float(x) for x in out)


def loss_gradient(image, target, rows=(0, 0)):
    image = np.ascontiguousarray(image, dtype=np.float64)
    target = np.ascontiguousarray(target, dtype=np.uint8)
    h, w = target.shape[:2]
    g = np.zeros((h, w, 3), dtype=np.float64)
    oracle().orc_loss_gradient(ptr(image), ptr(target), w, h, ptr(g), rows[0], rows[1])
    return g


def backward(proj, cam, offsets, ids, image, image_gradient, tile_range=(0, 0)):
    n = len(proj)
    g9 = np.zeros((9, n), dtype=np.float64)
    a2 = np.zeros((2, n), dtype=np.float64)
    ids = np.ascontiguousarray(ids, dtype=np.int32) if len(ids) else np.zeros(1, dtype=np.int32)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    image = np.ascontiguousarray(image, dtype=np.float64)
    image_gradient = np.ascontiguousarray(image_gradient, dtype=np.float64)
    oracle().orc_backward(ptr(proj), n, cam_ref(cam), ptr(offsets), ptr(ids), ptr(image), ptr(image_gradient),
                          ptr(g9), ptr(a2), tile_range[0], tile_range[1])
    return g9, a2


def projection_statistics(proj, cam, g9, a2):
    n = len(proj)
    stats = np.zeros((2, n), dtype=np.float64)
    abs_stats = np.zeros(n, dtype=np.float64)
    oracle().orc_projection_statistics(ptr(proj), n, cam_ref(cam), ptr(g9), ptr(a2), ptr(stats), ptr(abs_stats))
    return stats, abs_stats


def map_gradients(params, cam, sh_degree, g9):
    params = np.ascontiguousarray(params, dtype=np.float32)
    n = params.shape[1]
    g58 = np.zeros((58, n), dtype=np.float64)
    g9 = np.ascontiguousarray(g9, dtype=np.float64)
    oracle().orc_map_gradients(ptr(params), n, cam_ref(cam), sh_degree, ptr(g9), ptr(g58))
    return g58


def adam(params, m, v, g58, lr, step):
    lrs = LR(**lr)
    oracle().orc_adam(ptr(params), ptr(m), ptr(v), ptr(g58), params.shape[1], ctypes.byref(lrs), step)


def density_counts(params, grad_sums, abs_sums, obs, grad_thr, split_thr, min_opacity, max_world, prune_large,
                   abs_thr):
    params = np.ascontiguousarray(params, dtype=np.float32)
    n = params.shape[1]
    out = np.zeros((n, 4), dtype=np.int32)
    grad_sums = np.ascontiguousarray(grad_sums, dtype=np.float32)
    abs_sums = np.ascontiguousarray(abs_sums, dtype=np.float32)
    obs = np.ascontiguousarray(obs, dtype=np.uint32)
    oracle().orc_density_counts(ptr(params), n, ptr(grad_sums), ptr(abs_sums), ptr(obs), grad_thr, split_thr,
                                min_opacity, max_world, int(prune_large), abs_thr, ptr(out))
    return out


def density_apply(params, counts4, samples):
    params = np.ascontiguousarray(params, dtype=np.float32)
    n = params.shape[1]
    total = int(counts4[:, 0].sum() + counts4[:, 1].sum() + 2 * counts4[:, 3].sum())
    out = np.zeros((58, max(total, 1)), dtype=np.float32)
    parents = np.zeros(max(total, 1), dtype=np.int32)
    hist = np.zeros(max(total, 1), dtype=np.int32)
    counts4 = np.ascontiguousarray(counts4, dtype=np.int32)
    samples = np.ascontiguousarray(samples, dtype=np.float32)
    m = oracle().orc_density_apply(ptr(params), n, ptr(counts4), ptr(samples), ptr(out), ptr(parents), ptr(hist))
    return out[:, :m], parents[:m], hist[:m]


def knn3(points):
    points = np.ascontiguousarray(points, dtype=np.float32)
    n = points.shape[0]
    d = np.zeros(n, dtype=np.float64)
    nb = np.zeros((n, 3), dtype=np.int32)
    if n:
        oracle().orc_knn3(ptr(points), n, ptr(d), ptr(nb))
    return d, nb


def initial_parameters(points, colors, mean_dist2, initial_opacity=0.1):
    """The 58 x n parameter block GaussianSplatting::InitializeGaussians packs
    from a point cloud (gaussian_splatting.cpp:96-113), in float32 as the
    reference computes it: position rows 0-2 = the point; log-scale rows 3-5 =
    0.5 * log(max(mean_dist2, 1e-7)); axis-angle rows 6-8 = 0; opacity logit
    row 9 = log(0.1 / 0.9); SH DC rows 10, 26, 42 = (colour - 0.5) / C0 with
    C0 = 0.28209479177387814; every other SH row 0. mean_dist2 is the 3-NN mean
    squared distance of ComputeMeanDist2Cuda (knn.cu:180-255)."""
    pts = np.asarray(points, dtype=np.float32)
    col = np.asarray(colors, dtype=np.float32)
    d = np.asarray(mean_dist2, dtype=np.float32)
    n = pts.shape[0]
    out = np.zeros((58, n), dtype=np.float32)
    f32 = np.float32
    scale = (f32(0.5) * np.log(np.maximum(d, f32(1e-7)))).astype(np.float32)
    o = f32(initial_opacity)
    logit = np.log(o / (f32(1) - o)).astype(np.float32)
    for a in range(3):
        out[a] = pts[:, a]
        out[3 + a] = scale
        out[10 + 16 * a] = (col[:, a] - f32(0.5)) / f32(0.28209479177387814)
    out[9] = logit
    return out


def set_threads(k):
    return oracle().orc_set_threads(int(k))


# ---------------------------------------------------------------- learned density MLP
MLP_LAYOUT = dict(W1=(0, (64, 16)), b1=(1024, (64,)), W2=(1088, (64, 64)), b2=(5184, (64,)), W3=(5248, (4, 64)),
                  b3=(5504, (4,)))


def mlp_unpack(w):
    w = np.asarray(w, dtype=np.float64)
    return {k: w[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in MLP_LAYOUT.items()}


def mlp_forward(w, features):
    """FP64 forward of the 16 -> 64 -> 64 -> 4 ReLU MLP: (z1, h1, z2, h2, logits)."""
    p = mlp_unpack(w)
    f = np.asarray(features, dtype=np.float64)
    z1 = f @ p["W1"].T + p["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ p["W2"].T + p["b2"]
    h2 = np.maximum(z2, 0.0)
    return z1, h1, z2, h2, h2 @ p["W3"].T + p["b3"]


def mlp_loss_gradient(w, features, labels, sample_weights):
    """FP64 loss and gradient of sum_i (w_i / sum w) * CE(softmax(MLP(f_i)), label_i),
    the objective the GPU training kernels minimise; gradient in the flat weight
    layout of MLP_LAYOUT."""
    p = mlp_unpack(w)
    f = np.asarray(features, dtype=np.float64)
    z1, h1, z2, h2, lg = mlp_forward(w, f)
    lg = lg - lg.max(axis=1, keepdims=True)
    prob = np.exp(lg)
    prob /= prob.sum(axis=1, keepdims=True)
    nw = np.asarray(sample_weights, dtype=np.float64)
    nw = nw / nw.sum()
    idx = np.arange(f.shape[0])
    labels = np.asarray(labels)
    loss = -np.sum(nw * np.log(prob[idx, labels]))
    dl = prob.copy()
    dl[idx, labels] -= 1.0
    dl *= nw[:, None]
    g = {"W3": dl.T @ h2, "b3": dl.sum(0)}
    dz2 = (dl @ p["W3"]) * (z2 > 0)
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = (dz2 @ p["W2"]) * (z1 > 0)
    g["W1"], g["b1"] = dz1.T @ f, dz1.sum(0)
    out = np.zeros(5508)
    for k, (o, s) in MLP_LAYOUT.items():
        out[o:o + int(np.prod(s))] = g[k].ravel()
    return loss, out
