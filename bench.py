"""Benchmark of the 3DGS training hot path on B200.

One step = one training iteration of the plain FP32 form on the 1.2M-Gaussian
cap of the 1600x1064 ring-camera training scene: project + depth/tile ordering +
per-tile blend + fused L1/SSIM gradient + backward + chain rule + Adam, through
the library's C ABI (gs_native Renderer + Solver). This is the steady-state
iteration of the training schedule (iterations 15k-30k: SH degree 3, no
densification), with the model at the Gaussian cap.

Scene (seeded, synthetic): the hidden target model is 1.5M Gaussians (seed 7,
means N(0, 3^2)); 200 cameras on a ring of radius 8 at elevation +/-15 deg,
1600x1064, fx = fy = 1400, every tenth held out; targets are rendered from the
hidden model and quantised to u8. The model being optimised is a 1.2M-Gaussian
draw of the same distribution (seed 8).

Ten forms of the same iteration are timed, each from the same initial model:
`plain_fp32` (eager launches from the host, the reference-parity form),
`graph_fp32` (the iteration captured once as a CUDA graph over a fixed record
capacity and replayed from a device schedule of views), `culled_fp32` /
`culled_graph_fp32` (exact tile culling: only records whose tile the alpha
>= 1/255 ellipse reaches are emitted and sorted; images and gradients are
unchanged), `culled_sparse_fp32` / `culled_sparse_graph_fp32` (culling plus the
visibility-masked Adam step on the Morton-ordered model the trainer's spatial
order keeps - Gaussians outside the view keep p, m, v - and the fast blend
arithmetic) and
`precision_bf16_culled_sparse` / `..._graph` (all of that plus SH rows and their
Adam moments stored in bf16 with stochastic rounding and the tcgen05 SSIM; fp32
blending and accumulation) and `precision_bf16_fp32ssim_culled_sparse` /
`..._graph` (the same with the fp32 CUDA-core SSIM gradient). `value` is the fastest form that completed without a record
overflow; all are in `forms`, with `chosen_over_plain` the ratio to the plain
form. The held-out PSNR of each form's full training run is measured by
synthetic_run.py (the metric's 0.1 dB condition).

Printed JSON line: `value` is iterations/s with targets resident in HBM,
`e2e` the same through host buffers (every step uploads its target from pinned
host memory - the next step's upload overlapping the current step on a copy
stream - and copies its loss back to pinned memory, which the host reads two
steps later), plus per-stage device times, the roofline of the dominant
kernel and SM clocks sampled during the timed region. After the timed regions:
`reference_cuda`, the reference's own CUDA build (compiled unmodified) running
the steady-state loop of its trainer on the same workload; `psnr_gate`,
held-out PSNR of plain and chosen training runs on a reduced schedule (the
metric's 0.1 dB condition); and `cpu_baseline`, one full CPU training step
timed on the host cores (the reference's own test/cpu_reference.h forward and
loss, the FP64 oracle port for the gradients and Adam). `--impl reference`
times only that CPU implementation of the path.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "gs-native_b200")]

METRIC = "iters/sec @1.2M Gaussians 1600×1064: chosen form vs plain FP32, ΔPSNR≤0.1 dB"
UNIT = "iters/sec"
WORKLOAD = ("training step (render, L1+SSIM gradient, backward, Adam) at the 1.2M-Gaussian cap, 1600x1064, "
            "SH degree 3, one ring view per step")
SH_DEGREE = 3
TARGET_GAUSSIANS = 1_500_000
MODEL_GAUSSIANS = 1_200_000
# DRAM bytes (read + write) of one gaussian_update launch on this workload, per
# update form, from the ncu captures summarised in profiles/.
NCU_TRAFFIC = {
    "dense": (939_872_768 + 794_836_736,
              "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/gaussian_update_plain_1.2M.md"),
    "sparse": (615_015_680 + 483_678_208,
               "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/gaussian_update_sparse_1.2M.md"),
    "sparse_bf16": (380_198_656 + 268_296_960,
                    "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/gaussian_update_bf16_sparse_1.2M.md"),
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="gsn", choices=["gsn", "reference"])
    p.add_argument("--gaussians", type=int, default=MODEL_GAUSSIANS)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--profile-only", action="store_true",
                   help="warm-up steps plus one step on 3 views, no JSON (for ncu captures)")
    p.add_argument("--views", type=int, default=0, help="number of training views used (0 = all 180)")
    p.add_argument("--precision", action="store_true", help="with --profile-only: run the precision form")
    p.add_argument("--fp32-ssim", action="store_true",
                   help="with --profile-only --precision: the fp32 SSIM gradient instead of the tcgen05 one")
    p.add_argument("--culled", action="store_true", help="with --profile-only: exact tile culling on")
    p.add_argument("--sparse", action="store_true", help="with --profile-only: sparse Adam on the Morton-ordered model")
    p.add_argument("--multiview", action="store_true", help="with --profile-only: the 32-view multi-view render")
    p.add_argument("--no-multiview", action="store_true", help="skip the 32-view multi-view measurement")
    p.add_argument("--no-reference-cuda", action="store_true", help="skip the reference CUDA build's leg")
    p.add_argument("--no-psnr-gate", action="store_true", help="skip the held-out PSNR gate runs")
    p.add_argument("--no-large-scene", action="store_true",
                   help="skip the 3.0M-Gaussian 2048x1360 batched-form measurement")
    p.add_argument("--gate-iterations", type=int, default=6000,
                   help="iterations of each held-out PSNR gate run (reduced schedule)")
    p.add_argument("--no-programmatic-launch", action="store_true",
                   help="launch the step's kernels without programmatic dependent launch (for comparison)")
    return p.parse_args()


def position_lr(iteration, extent):
    f = min(1.0, iteration / 30000.0)
    return extent * math.exp(math.log(1.6e-4) * (1 - f) + math.log(1.6e-6) * f)


def scene(n_model):
    import scenes
    target = scenes.random_gaussians(TARGET_GAUSSIANS, 7, mean_sigma=3.0)
    model = scenes.random_gaussians(n_model, 8, mean_sigma=3.0)
    train, _ = scenes.training_scene_cameras()
    centers = []
    for c in train:
        R = np.array(list(c.R_c_w), dtype=np.float64).reshape(3, 3)
        t = np.array(list(c.t_c_w), dtype=np.float64)
        centers.append(-R.T @ t)
    centers = np.array(centers)
    extent = 1.1 * np.linalg.norm(centers - centers.mean(0), axis=1).max()
    return target, model, train, float(extent)


class ClockSampler:
    """nvidia-smi SM clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.rows = []
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(device_index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        if not self.rows:
            return None
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[4 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def algorithmic_bytes(n, records, tiles, pixels, s=16, tile_passes=2, visible=None, culled=False, sparse=False,
                      bf16=False):
    """Compulsory HBM bytes per launch of each stage for a form (N Gaussians, V
    visible, R records, T tiles, P pixels): culled records are emitted with their conic (36 B per visible
    Gaussian), the sparse update moves only visible Gaussians' rows, the
    precision layout stores the 48 SH rows in 2 bytes."""
    vis = n if visible is None else visible
    sh_bytes = 2 if bf16 else 4
    row_bytes = 10 * 4 + 3 * s * sh_bytes              # one Gaussian's parameter rows
    updated = vis if sparse else n
    return {
        "project": n * (row_bytes + 68),
        "depth_sort": 4 * n * 20,
        "record_scan": n * 20,
        "emit_records": records * 8 + vis * (36 if culled else 24),
        "tile_sort": tile_passes * records * 20,
        "tile_ranges": records * 4 + (tiles + 1) * 8,
        "raster_forward": records * 40 + pixels * 16,
        "loss_gradient": pixels * 3 * 9,
        "raster_backward": records * 40 + pixels * 28 + vis * 48,
        "gaussian_update": updated * row_bytes * 6 + n * (48 + 4 + 16),
    }


# FP32 operations per (pixel, record) pair the blend takes, counting an FMA as
# two: forward 16 (offset, two-FMA power, exp2, clamp, transmittance FMA, weight,
# three colour FMAs); backward 46 (offset, power, exp2, clamp, weight, 1 - alpha
# and its reciprocal, dL/dC . c, dL/dalpha, three colour-gradient FMAs, the
# chain to the power, d(mean) and d(conic) accumulations, |d mean| sums, the
# carried colour and transmittance). Counted from the fast form's arithmetic.
FLOP_PER_PAIR = {"raster_forward": 16, "raster_backward": 46}
# No FP32 figure is measured for this pool; the nominal FMA rate at the
# maximum SM clock: 148 SMs x 128 lanes x 2 FLOP x 1.965 GHz.
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def cpu_step(oracle, params64, m, v, cam, target_u8, lr, step, use_reference):
    """One full CPU training step on the whole frame (no sampling), legs timed:
    the forward render and the loss value by the reference's own CPU reference
    (test/cpu_reference.h RenderReference + ComputeLoss, single-threaded as
    written) when `use_reference`, else by the FP64 oracle; projection, tile
    lists, loss gradient, backward, chain rule and Adam by the FP64 oracle port
    on its OpenMP threads (the reference has no CPU backward)."""
    legs = {}
    t = time.perf_counter()
    p32 = params64.astype(np.float32)
    proj = oracle.project(p32, cam, SH_DEGREE)
    offsets, ids = oracle.tile_lists(proj, cam)
    legs["project_and_lists"] = time.perf_counter() - t
    t = time.perf_counter()
    if use_reference:
        image = oracle.ref_cpu_render(p32, cam, [0, 0, 0], SH_DEGREE)
        loss = oracle.ref_cpu_loss(image, target_u8)
    else:
        image, _, _ = oracle.render(proj, cam, offsets, ids, [0, 0, 0])
        loss = oracle.loss(image, target_u8)
    legs["forward_and_loss"] = time.perf_counter() - t
    t = time.perf_counter()
    gI = oracle.loss_gradient(image, target_u8)
    g9, _ = oracle.backward(proj, cam, offsets, ids, image, gI)
    g58 = oracle.map_gradients(p32, cam, SH_DEGREE, g9)
    oracle.adam(params64, m, v, g58, lr, step)
    legs["gradients_and_adam"] = time.perf_counter() - t
    return legs, loss


def cpu_baseline(model, cam, target_u8, extent, steps=1, budget_s=None, threads=None):
    """Full training steps on the CPU (see cpu_step) over the whole frame:
    `steps` of them, or as many as fit in `budget_s` seconds (at least one).
    Returns the rate, the steps actually run and the per-leg seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cores = threads or len(os.sched_getaffinity(0))
    oracle.set_threads(cores)
    use_reference = oracle.ref_cpu_available()
    n = model.shape[1]
    params64 = model.astype(np.float64)
    m = np.zeros_like(params64)
    v = np.zeros_like(params64)
    lr = dict(oracle.REFERENCE_LR)
    lr["position"] = position_lr(15000, extent)
    per_step, legs_all = [], []
    t0 = time.perf_counter()
    for step in range(steps):
        a = time.perf_counter()
        legs, _ = cpu_step(oracle, params64, m, v, cam, target_u8, lr, step + 1, use_reference)
        per_step.append(time.perf_counter() - a)
        legs_all.append(legs)
        if budget_s is not None and time.perf_counter() - t0 + per_step[-1] > budget_s:
            break
    total = sum(per_step)
    run = len(per_step)
    legs = {k: round(float(np.mean([l[k] for l in legs_all])), 3) for k in legs_all[0]}
    fwd = ("RenderReference + ComputeLoss of the reference's test/cpu_reference.h (compiled unmodified "
           "against an OpenCV shim), single-threaded as written" if use_reference else
           "FP64 oracle render and loss (the reference's CPU reference was not built)")
    return {"value": run / total, "unit": UNIT, "cores": cores, "kind": "reference" if use_reference else "port",
            "sample": (f"{run} full training step(s) of the whole 1600x1064 frame on {n} Gaussians, no sampling "
                       f"or scaling: forward and loss by {fwd}; projection, tile lists, loss gradient, backward, "
                       f"chain rule and Adam by the FP64 oracle port on {cores} threads"),
            "threads": {"forward_and_loss": 1 if use_reference else cores, "port": cores},
            "legs_s": legs, "steps_run": run, "seconds": round(total, 2)}


def measure_reference_cuda(gsn, torch, model, train, targets, lr, args):
    """The reference's own CUDA build (renderer.cu + solver.cu compiled
    unmodified for sm_100a into oracle/_ref/libgsref.so) on the same workload
    as the forms: the steady-state loop of GaussianSplatting::Train (Render +
    Iterate per step, no log line) from the same initial model and views, with
    the targets resident in HBM (`value`) and uploaded from pageable host
    memory with cudaMemcpy2D every step as Train does (`e2e`). Timed by CUDA
    events around the loop inside the harness (no Python in the loop). This is
    a baseline leg: it runs after, and outside, the timed regions of the
    library's forms."""
    import ctypes
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_available():
        return {"unavailable": "oracle/_ref/libgsref.so was not built (no reference tree where build() ran)"}
    V, I, F, P = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.POINTER
    r, s = V(), V()
    oracle.ref_fn("ref_renderer_create", [P(V)])(ctypes.byref(r))
    oracle.ref_fn("ref_solver_create", [P(V)])(ctypes.byref(s))
    replay = oracle.ref_fn("ref_train_replay", [V, V, V, I, V, V, I, V, V, V, V, V, F, I, P(F)])
    n = model.shape[1]
    p = torch.from_numpy(np.ascontiguousarray(model)).cuda()
    img = torch.empty((1064, 1600, 3), device="cuda")
    tbuf = torch.empty((1064, 1600, 3), dtype=torch.uint8, device="cuda")
    cams = (gsn.Camera * len(train))(*train)
    bg = (ctypes.c_float * 3)(0, 0, 0)
    warm = [k % len(train) for k in range(args.warmup)]
    views = [(args.warmup + k) % len(train) for k in range(args.steps)]
    # pageable host copies of the targets the timed steps use (the reference
    # trainer keeps its images in cv::Mat host memory)
    pageable = {v: np.ascontiguousarray(targets[v].cpu().numpy()) for v in set(views)}
    hptr = (V * len(train))(*[pageable[v].ctypes.data if v in pageable else None for v in range(len(train))])

    def run(vs, host):
        arr = (I * len(vs))(*vs)
        ms = F()
        torch.cuda.synchronize()
        st = replay(r, s, V(p.data_ptr()), n, cams, arr, len(vs), hptr if host else None,
                    V(0) if host else V(targets.data_ptr()), V(tbuf.data_ptr()), bg, V(img.data_ptr()), lr,
                    SH_DEGREE, ctypes.byref(ms))
        torch.cuda.synchronize()
        assert st == 0, f"reference replay failed ({st})"
        return ms.value

    # warm-up: the reference's renderer reallocates its record buffers at
    # exactly the new size whenever a frame has more records than any before,
    # and the record counts creep up as the model trains, so it first runs the
    # timed views twice (its buffers reach their steady size outside the
    # timed loops)
    run(warm, False)
    run(views, False)
    run(views, False)
    ms = run(views, False)
    ms_e2e = run(views, True)
    oracle.ref_fn("ref_solver_destroy", [V])(s)
    oracle.ref_fn("ref_renderer_destroy", [V])(r)
    return {"value": round(args.steps / (ms / 1000.0), 3), "ms_per_step": round(ms / args.steps, 4),
            "e2e": round(args.steps / (ms_e2e / 1000.0), 3), "e2e_ms_per_step": round(ms_e2e / args.steps, 4),
            "steps": args.steps, "warmup": args.warmup,
            "build": "renderer.cu + solver.cu compiled unmodified for sm_100a (oracle/_ref/libgsref.so)",
            "loop": ("GaussianSplatting::Train steady state: Render + Solver::Iterate per step, same initial "
                     "1.2M model, views and position learning rate as the forms; per-iteration log line off")}


def measure_multiview(gsn, torch, model, stream, sp, args, world):
    """32 views of uneven resolution (640x480 ... 2560x1440, sphere of radius 10,
    seed 23) of the 1.2M model: frames/s of the unbatched single-view path
    (one Render per view, record count read back per view) against one
    multi-view render (per-view ordering, one persistent blend launch) in the
    configuration the autotuner picks on the same views."""
    import scenes
    cams = scenes.multiview_cameras(32, seed=23)
    p = torch.from_numpy(model).cuda()
    n = p.shape[1]
    imgs = [torch.empty((c.height, c.width, 3), device="cuda") for c in cams]
    ptrs = [x.data_ptr() for x in imgs]
    reps = 3
    single = gsn.Renderer()
    single.set_stream(sp)

    def unbatched():
        for c, x in zip(cams, imgs):
            assert single.render(p.data_ptr(), n, c, [0, 0, 0], x.data_ptr(), SH_DEGREE) == 0

    mv = gsn.MultiView()
    mv.set_stream(sp)
    rows = mv.autotune(p.data_ptr(), n, cams, ptrs, [0, 0, 0], SH_DEGREE, repeats=2)

    def batched():
        mv.render(p.data_ptr(), n, cams, ptrs, [0, 0, 0], SH_DEGREE)

    def time(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_single = time(unbatched)
    ms_multi = time(batched)
    sizes = {}
    for c in cams:
        sizes[f"{c.width}x{c.height}"] = sizes.get(f"{c.width}x{c.height}", 0) + 1
    best = mv.config()
    return {"views": len(cams), "resolutions": sizes, "gaussians": n,
            "unbatched_frames_per_s": round(world * 1000.0 * len(cams) / ms_single, 2),
            "batched_frames_per_s": round(world * 1000.0 * len(cams) / ms_multi, 2),
            "speedup": round(ms_single / ms_multi, 3),
            "config": {"tile_w": best[0], "tile_h": best[1], "threads": best[2], "key_bits": best[3]},
            "autotune_ms": [[r["tile_w"], r["tile_h"], r["threads"], r["key_bits"], round(r["ms"], 3)] for r in rows]}


def measure_large_scene(gsn, torch, stream, sp, args, world):
    """The batched form at the large scene's scale: a 3.0M-Gaussian model (seed
    12, means N(0, 4^2)) trained against targets rendered from the hidden
    4M-Gaussian model (seed 11, means N(0, 4^2)) on 20 of the 300 two-ring
    views (radii 8 and 12, 2048x1360, fx = fy = 1800). Iterations/s of the
    unbatched, un-captured plain FP32 path against the chosen form (bf16 SH,
    exact culling, sparse Adam on the Morton order, fast blend arithmetic, one
    CUDA graph per step over a fixed record capacity), and the 32-view
    multi-view render of the same model."""
    import scenes
    hidden = scenes.random_gaussians(4_000_000, 11, mean_sigma=4.0)
    model = scenes.random_gaussians(3_000_000, 12, mean_sigma=4.0)
    cams = scenes.two_ring_cameras()
    views = cams[::15][:20]
    W, H = views[0].width, views[0].height
    centers = np.array([-np.array(list(c.R_c_w)).reshape(3, 3).T @ np.array(list(c.t_c_w)) for c in cams])
    extent = 1.1 * float(np.linalg.norm(centers - centers.mean(0), axis=1).max())
    lr = position_lr(15000, extent)
    img = torch.empty((H, W, 3), device="cuda")
    targets = torch.empty((len(views), H, W, 3), dtype=torch.uint8, device="cuda")
    hp = torch.from_numpy(hidden).cuda()
    maker = gsn.Renderer()
    maker.set_stream(sp)
    for k, c in enumerate(views):
        assert maker.render(hp.data_ptr(), hp.shape[1], c, [0, 0, 0], img.data_ptr(), SH_DEGREE) == 0
        targets[k] = (img * 255.0).round().clamp(0, 255).to(torch.uint8)
    del hp, maker
    torch.cuda.empty_cache()
    n = model.shape[1]

    def make(chosen):
        r, s = gsn.Renderer(), gsn.Solver()
        r.set_stream(sp)
        s.set_stream(sp)
        block = model
        if chosen:
            r.set_exact_culling(True)
            r.set_fast_blend(True)
            r.set_bf16_sh(True)
            s.set_sparse_adam(True)
            s.set_bf16_sh(True)
            s.set_tensor_core_loss(False)
            dev_model = torch.from_numpy(model).cuda()
            perm = torch.empty(n, dtype=torch.int32, device="cuda")
            gsn.spatial_permutation(dev_model.data_ptr(), n, perm.data_ptr(), sp)
            block = dev_model[:, perm.long()].cpu().numpy()
            del dev_model, perm
            params = gsn.to_precision_layout(block, torch)
        else:
            params = torch.from_numpy(np.ascontiguousarray(block)).cuda()
        return r, s, params

    def step(r, s, params, k):
        c = views[k % len(views)]
        assert r.render(params.data_ptr(), n, c, [0, 0, 0], img.data_ptr(), SH_DEGREE) == 0
        assert s.iterate(c, r, img.data_ptr(), targets[k % len(views)].data_ptr(), params.data_ptr(), n, lr,
                         SH_DEGREE) == 0

    def timed(run):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    r, s, params = make(False)
    for k in range(args.warmup):
        step(r, s, params, k)
    ms_plain = timed(lambda: [step(r, s, params, args.warmup + k) for k in range(args.steps)])
    records_plain = int(r.buffers().record_count_host)
    del r, s, params
    torch.cuda.empty_cache()
    r, s, params = make(True)
    for k in range(args.warmup):
        step(r, s, params, k)
    torch.cuda.synchronize()
    records = int(r.buffers().record_count_host)
    graph = gsn.Graph()
    capacity = int(records * 1.5) + 65536
    graph.capture(r, s, params.data_ptr(), n, views, targets.data_ptr(), W * H * 3, [0, 0, 0], img.data_ptr(),
                  SH_DEGREE, capacity, sp)
    schedule = [(args.warmup + k) % len(views) for k in range(args.steps)]
    graph.run(schedule[:max(3, args.warmup)], [lr] * max(3, args.warmup))
    ms_graph = timed(lambda: graph.run(schedule, [lr] * len(schedule)))
    status = graph.check()
    graph.close()
    del r, s, params, targets
    torch.cuda.empty_cache()
    rate = lambda t: round(job_rate(world, args.steps, t), 3)  # noqa: E731
    multiview = measure_multiview(gsn, torch, model, stream, sp, args, world)
    return {"gaussians": n, "hidden_gaussians": hidden.shape[1], "resolution": [W, H], "views": len(views),
            "plain_fp32_eager": {"value": rate(ms_plain), "ms_per_step": round(ms_plain / args.steps, 4),
                                 "records_per_step": records_plain},
            "chosen_graph": {"value": rate(ms_graph), "ms_per_step": round(ms_graph / args.steps, 4),
                             "record_capacity": capacity, "records_per_step": records, "status": status},
            "chosen_over_plain": round(ms_plain / ms_graph, 4), "multiview": multiview}


def run_reference(args):
    """The CPU implementation of the path on the host cores (rank 0 only): full
    training steps of the bench workload (cpu_step: the reference's own
    test/cpu_reference.h forward and loss, the FP64 oracle port for the rest)
    for as many of the requested steps as fit in about 90 s (at least one). No
    warm-up steps are run: CPU code has nothing to warm across steps of ~15 s.
    The line reports the steps actually run."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    target_model, model, train, extent = scene(args.gaussians)
    cam = train[0]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    img = oracle.render_params(target_model, cam, [0, 0, 0], SH_DEGREE)
    target = np.clip(np.rint(img * 255), 0, 255).astype(np.uint8)
    steps = max(1, args.steps)
    res = cpu_baseline(model, cam, target, extent, steps=steps, budget_s=90.0)
    value = res["value"]
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": res["steps_run"], "warmup": 0, "requested": {"steps": args.steps, "warmup": args.warmup},
        "ms_per_step": 1000.0 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "form": "CPU: reference test/cpu_reference.h forward + loss, FP64 port "
                                                 "for the gradients and Adam",
                   "gaussians": args.gaussians, "width": 1600, "height": 1064, "sampling": "none (whole frame)"},
        "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample", "threads", "legs_s")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def reduce_max_over_ranks(dist, value, device):
    """The largest of every rank's value (each rank's device time of the same
    timed region, so the job is timed by its slowest rank); the value itself
    without a process group."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, steps_per_rank, ms):
    """Whole-job iterations per second: every rank runs its own steps (replicas,
    weak scaling) and the job takes the slowest rank's `ms`."""
    return world * steps_per_rank / (ms / 1000.0)


def run_gsn(args):
    import torch
    import gsn
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    gsn.lib()
    gsn.set_programmatic_launch(not args.no_programmatic_launch)
    target_model, model, train, extent = scene(args.gaussians)
    views = 3 if args.profile_only else args.views
    if views:
        train = train[:views]
    n = model.shape[1]
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    # hidden-model targets, resident in HBM and in pinned host memory
    tm = torch.from_numpy(target_model).cuda()
    img = torch.empty((1064, 1600, 3), device="cuda")
    targets = torch.empty((len(train), 1064, 1600, 3), dtype=torch.uint8, device="cuda")
    maker = gsn.Renderer()
    for k, cam in enumerate(train):
        assert maker.render(tm.data_ptr(), tm.shape[1], cam, [0, 0, 0], img.data_ptr(), SH_DEGREE) == 0
        targets[k] = (img * 255.0).round().clamp(0, 255).to(torch.uint8)
    del tm, maker
    host_targets = targets.cpu().pin_memory()
    # end-to-end runs upload every step's target from pinned host memory; the
    # upload of step k + 1 runs on a copy stream into the other staging buffer
    # while step k computes (as a training loop prefetches its next input)
    # and each step's loss is copied back into a pinned ring the host reads two
    # steps later (it waits for step k - 2 before issuing step k + 1's upload)
    ring = 3
    staging = [torch.empty((1064, 1600, 3), dtype=torch.uint8, device="cuda") for _ in range(ring)]
    copy_stream = torch.cuda.Stream()
    ready = [torch.cuda.Event() for _ in range(ring)]
    done = [torch.cuda.Event() for _ in range(ring)]
    loss_ring = torch.zeros((ring, 4), dtype=torch.float64).pin_memory()
    e2e_seen = []
    lr = position_lr(15000, extent)
    loss_host = torch.zeros(4, dtype=torch.float64).pin_memory()

    class Form:
        """One form of the iteration: its own renderer, solver and parameter block."""

        def __init__(self, bf16, culled=False, sparse=False, tc_loss=True):
            self.renderer, self.solver = gsn.Renderer(), gsn.Solver()
            self.renderer.set_stream(sp)
            self.solver.set_stream(sp)
            self.renderer.set_exact_culling(culled)
            self.solver.set_sparse_adam(sparse)
            # the sparse forms already leave the reference's arithmetic: they also
            # take the fast blend arithmetic (Horner power, hardware exp2)
            self.renderer.set_fast_blend(sparse)
            block = model
            if sparse:
                # the trainer's spatial order (Morton order of the means after every
                # density step) - the order of the steady-state model it trains
                dev_model = torch.from_numpy(model).cuda()
                perm = torch.empty(n, dtype=torch.int32, device="cuda")
                gsn.spatial_permutation(dev_model.data_ptr(), n, perm.data_ptr(), sp)
                block = dev_model[:, perm.long()].cpu().numpy()
                del dev_model, perm
            if bf16:
                self.renderer.set_bf16_sh(True)
                self.solver.set_bf16_sh(True)
                self.solver.set_tensor_core_loss(tc_loss)
                self.params = gsn.to_precision_layout(block, torch)
            else:
                self.params = torch.from_numpy(np.ascontiguousarray(block)).cuda()

    upload_view = [0]  # view offset of the run being uploaded

    def upload(dst, k, buf):
        """Pinned-host upload of step k's target into dst on the copy stream."""
        with torch.cuda.stream(copy_stream):
            dst.copy_(host_targets[(upload_view[0] + k) % len(train)], non_blocking=True)
            ready[buf].record(copy_stream)

    def step(f, k, tgt=None):
        cam = train[k % len(train)]
        if tgt is None:
            tgt = targets[k % len(train)]
        assert f.renderer.render(f.params.data_ptr(), n, cam, [0, 0, 0], img.data_ptr(), SH_DEGREE) == 0
        assert f.solver.iterate(cam, f.renderer, img.data_ptr(), tgt.data_ptr(), f.params.data_ptr(), n, lr,
                                SH_DEGREE) == 0

    def read_loss(f, b):
        """Async D2H copy of the step's loss into ring slot b, marked by done[b]."""
        gsn.memcpy_async(loss_ring[b].data_ptr(), f.solver.loss_device(), 32, sp)
        done[b].record(stream)

    def pipelined(steps, dst, issue):
        """Every step uploads its target (dst(k): device buffer of step k) and
        reads its loss back; the host waits for step k - 2 (its loss) before
        reusing that step's slot for step k + 1's upload."""
        upload(dst(0), 0, 0)
        for k in range(steps):
            b = k % ring
            if k + 1 < steps:
                nb = (k + 1) % ring
                if k + 1 >= ring:
                    done[nb].synchronize()
                    e2e_seen.append(float(loss_ring[nb, 3]))
                upload(dst(k + 1), k + 1, nb)
            stream.wait_event(ready[b])
            issue(k, b)
        stream.synchronize()
        e2e_seen.extend(float(loss_ring[(k % ring), 3]) for k in range(max(0, steps - ring), steps))
        loss_host.copy_(loss_ring[(steps - 1) % ring])

    def e2e_steps(f, k0):
        """Steps through host buffers (see pipelined)."""
        def run(steps):
            def issue(k, b):
                step(f, k0 + k, staging[b])
                read_loss(f, b)
            pipelined(steps, lambda k: staging[k % ring], issue)
        return run

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(ms):
        return reduce_max_over_ranks(dist, ms, "cuda")

    def timed(run, steps):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = gsn.launch_count()
        e0.record(stream)
        run(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        launches = gsn.launch_count() - launches0
        barrier()
        return max_over_ranks(e0.elapsed_time(e1)), launches

    def eager_steps(f, k0):
        return lambda steps: [step(f, k0 + k) for k in range(steps)]

    def profile_stages(f):
        gsn.profile_enable(True)
        for k in range(args.steps):
            step(f, args.warmup + k)
        st = gsn.profile_collect()
        gsn.profile_enable(False)
        return {k: v / args.steps for k, v in st.items() if v > 0}

    def count_pairs(f):
        """(pixel, record) pairs the blend takes per step, over the timed steps'
        views (a counting pass after the timed regions)."""
        counter = torch.zeros(1, dtype=torch.int64, device="cuda")
        f.renderer.set_pair_counter(counter.data_ptr())
        for k in range(args.steps):
            step(f, args.warmup + k)
        f.renderer.set_pair_counter(0)
        torch.cuda.synchronize()
        return float(counter.item()) / args.steps

    def measure(f, with_stages=True):
        """Eager timing, per-stage profile, end-to-end timing, then the graph form."""
        for k in range(args.warmup):
            step(f, k)
        torch.cuda.synchronize()
        ms, launches = timed(eager_steps(f, args.warmup), args.steps)
        stages = profile_stages(f) if with_stages else None
        if stages is not None:
            stages["pairs_per_step"] = count_pairs(f)
        f.solver.set_compute_loss(True)
        upload_view[0] = 0
        e2e_steps(f, 0)(2)
        upload_view[0] = args.warmup
        ms_e2e, _ = timed(e2e_steps(f, args.warmup), args.steps)
        records = int(f.renderer.buffers().record_count_host)
        # visible Gaussians of the last frame, read while the renderer is alive
        counts = torch.empty(n, dtype=torch.int32, device="cuda")
        gsn.memcpy(counts.data_ptr(), f.renderer.buffers().tile_counts, 4 * n)
        visible_count = int((counts > 0).sum().item())
        # batched form: the iteration captured once as a CUDA graph over a fixed
        # record capacity, replayed from a device schedule of views
        graph = gsn.Graph()
        capacity = int(records * 1.5) + 65536
        graph.capture(f.renderer, f.solver, f.params.data_ptr(), n, train, targets.data_ptr(), 1064 * 1600 * 3,
                      [0, 0, 0], img.data_ptr(), SH_DEGREE, capacity, sp)
        schedule = [(args.warmup + k) % len(train) for k in range(args.steps)]
        graph.run(schedule[:max(3, args.warmup)], [lr] * max(3, args.warmup))
        ms_graph, graph_launches = timed(lambda steps: graph.run(schedule[:steps], [lr] * steps), args.steps)
        status = graph.check()

        def graph_e2e(steps):
            # one replay per step; the uploads go straight into the view's resident
            # slot (the steps in flight use other views: the schedule cycles 180)
            def issue(k, b):
                graph.run([schedule[k]], [lr])
                read_loss(f, b)
            upload_view[0] = args.warmup  # schedule[k] = (warmup + k) % views
            pipelined(steps, lambda k: targets[schedule[k]], issue)

        ms_graph_e2e, _ = timed(graph_e2e, args.steps)
        status = status or graph.check()
        per_step = graph.launches_per_step()
        graph.close()
        rate = lambda t: job_rate(world, args.steps, t)  # noqa: E731
        eager = {"value": round(rate(ms), 3), "ms_per_step": round(ms / args.steps, 4), "e2e": round(rate(ms_e2e), 3),
                 "gpu_launches": int(launches), "psnr_db_last_step": round(float(loss_host[3]), 3)}
        graphed = {"value": round(rate(ms_graph), 3), "ms_per_step": round(ms_graph / args.steps, 4),
                   "e2e": round(rate(ms_graph_e2e), 3), "gpu_launches": int(graph_launches),
                   "launches_per_step": per_step, "record_capacity": capacity, "status": status,
                   "psnr_db_last_step": round(float(loss_host[3]), 3)}
        return eager, graphed, stages, records, visible_count

    if args.profile_only:
        if args.multiview:
            # the 32-view persistent render in the default configuration, warmup + 1 times
            import scenes
            cams = scenes.multiview_cameras(32, seed=23)
            p = torch.from_numpy(model).cuda()
            imgs = [torch.empty((c.height, c.width, 3), device="cuda") for c in cams]
            mv = gsn.MultiView()
            mv.set_stream(sp)
            for _ in range(args.warmup + 1):
                mv.render(p.data_ptr(), n, cams, [x.data_ptr() for x in imgs], [0, 0, 0], SH_DEGREE)
            torch.cuda.synchronize()
            return
        f = Form(args.precision, args.culled, args.sparse, tc_loss=not args.fp32_ssim)
        for k in range(args.warmup + 1):
            step(f, k)
        torch.cuda.synchronize()
        return

    visible = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    smi_index = visible.split(",")[local] if visible else str(local)
    sampler = ClockSampler(smi_index) if rank == 0 else None
    plain = Form(False)
    plain_eager, plain_graph, stages, records, vis = measure(plain)
    del plain
    torch.cuda.empty_cache()
    culled = Form(False, True)
    culled_eager, culled_graph, culled_stages, culled_records, _ = measure(culled)
    del culled
    torch.cuda.empty_cache()
    sparse = Form(False, True, True)
    sparse_eager, sparse_graph, sparse_stages, _, _ = measure(sparse)
    del sparse
    torch.cuda.empty_cache()
    prec = Form(True, True, True)
    prec_eager, prec_graph, prec_stages, _, _ = measure(prec)
    del prec
    torch.cuda.empty_cache()
    prec32 = Form(True, True, True, tc_loss=False)
    prec32_eager, prec32_graph, prec32_stages, _, _ = measure(prec32, with_stages=True)
    clocks = sampler.stop() if sampler else None
    del prec32
    value = plain_eager["value"]
    ms = plain_eager["ms_per_step"] * args.steps
    psnr = plain_eager["psnr_db_last_step"]
    multiview = None if args.no_multiview else measure_multiview(gsn, torch, model, stream, sp, args, world)
    target0 = targets[0].cpu().numpy()
    # baselines and the accuracy gate, after (and outside) every timed region of the forms
    ref_cuda = None
    if not args.no_reference_cuda and world == 1:
        ref_cuda = measure_reference_cuda(gsn, torch, model, train, targets, lr, args)
    large = None
    if not args.no_large_scene and world == 1:
        large = measure_large_scene(gsn, torch, stream, sp, args, world)
    gate = None
    if not args.no_psnr_gate and world == 1:
        import synthetic_run
        torch.cuda.empty_cache()
        gate = synthetic_run.psnr_gate(torch, iterations=args.gate_iterations)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    cam = train[0]
    tiles = cam.tile_count_x * cam.tile_count_y
    pixels = cam.width * cam.height
    tile_bits = max(1, (tiles - 1).bit_length())
    passes = (tile_bits + 7) // 8
    alg = algorithmic_bytes(n, records, tiles, pixels, tile_passes=passes, visible=vis)
    peak, peak_kind = load_peaks()
    stage_table = {}
    for name, t in stages.items():
        if name == "pairs_per_step":
            continue
        entry = {"ms": round(t, 4)}
        if name in alg:
            gbs = alg[name] / (t / 1000.0) / 1e9
            entry.update(bytes=int(alg[name]), gbs=round(gbs, 1), hbm_frac=round(gbs / peak, 4))
        stage_table[name] = entry
    forms = {"plain_fp32": plain_eager, "graph_fp32": plain_graph, "culled_fp32": culled_eager,
             "culled_graph_fp32": culled_graph, "culled_sparse_fp32": sparse_eager,
             "culled_sparse_graph_fp32": sparse_graph, "precision_bf16_culled_sparse": prec_eager,
             "precision_bf16_culled_sparse_graph": prec_graph,
             "precision_bf16_fp32ssim_culled_sparse": prec32_eager,
             "precision_bf16_fp32ssim_culled_sparse_graph": prec32_graph}
    valid = {k: v for k, v in forms.items() if v.get("status", 0) == 0}
    chosen = max(valid, key=lambda k: valid[k]["value"])

    def stages_of(form):
        culled_f, sparse_f, bf16_f = "culled" in form, "sparse" in form, form.startswith("precision")
        return (prec32_stages if "fp32ssim" in form else prec_stages) if bf16_f else \
            sparse_stages if sparse_f else culled_stages if culled_f else stages

    def blend_roofline(form):
        """FP32 roofline of the blend kernels of a form: algorithmic FLOPs (the
        pairs the blend took this step x FLOP_PER_PAIR) over the kernel's
        per-step device time, against the nominal FP32 rate."""
        st = stages_of(form)
        pairs = st.get("pairs_per_step")
        out = {}
        for k in ("raster_backward", "raster_forward"):
            if k in st and pairs:
                ach = pairs * FLOP_PER_PAIR[k] / (st[k] / 1000.0) / 1e12
                out[k] = {"bound": "fp32", "kernel": k, "form": form, "achieved": round(ach, 3),
                          "peak": round(FP32_NOMINAL_TFLOPS, 1), "unit": "TFLOP/s",
                          "frac": round(ach / FP32_NOMINAL_TFLOPS, 4), "ms": round(st[k], 4),
                          "pairs_per_step": int(pairs), "flop_per_pair": FLOP_PER_PAIR[k],
                          "peak_source": ("nominal FP32 FMA rate, 148 SMs x 128 lanes x 2 FLOP x 1.965 GHz "
                                          "(MEASURED_PEAKS.json holds no FP32 figure)")}
        return out

    def roofline_of(form):
        """Roofline of the largest HBM-bound stage of a form, from its live stage times."""
        culled_f, sparse_f, bf16_f = "culled" in form, "sparse" in form, form.startswith("precision")
        st = stages_of(form)
        rec = culled_records if culled_f else records
        ab = algorithmic_bytes(n, rec, tiles, pixels, tile_passes=passes, visible=vis, culled=culled_f,
                               sparse=sparse_f, bf16=bf16_f)
        kernel_stages = {k: v for k, v in st.items() if k in ab}
        hbm = {k: v for k, v in kernel_stages.items() if k in ("gaussian_update", "project", "depth_sort",
                                                                "tile_sort", "emit_records", "loss_gradient")}
        top = max(hbm, key=hbm.get)
        achieved = ab[top] / (st[top] / 1000.0) / 1e9
        traffic = None
        if top == "gaussian_update" and n == MODEL_GAUSSIANS and (sparse_f or not bf16_f):
            traffic = NCU_TRAFFIC[("sparse_bf16" if bf16_f else "sparse") if sparse_f else "dense"]
        return {"bound": "hbm", "kernel": top, "form": form, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "algorithmic_bytes": int(ab[top]),
                "traffic": traffic[0] if traffic else None, "traffic_source": traffic[1] if traffic else None,
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured" else
                "fallback 6650 GB/s",
                "dominant_kernel": max(kernel_stages, key=kernel_stages.get),
                "dominant_note": ("the per-tile blend kernels are bound by the FP32/MUFU issue rate and the "
                                  "atomics of the backward, not by HBM; their HBM fractions are in `stages`")}

    roofline = roofline_of(chosen)
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        res = cpu_baseline(model, train[0], target0, extent, steps=1)
        cpu = {k: res[k] for k in ("value", "unit", "cores", "kind", "sample", "threads", "legs_s")}
    out = {
        "metric": METRIC, "value": forms[chosen]["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": forms[chosen]["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32" if chosen.startswith("precision") else "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD,
                   "form": chosen, "gaussians": n, "width": 1600, "height": 1064,
                   "records_per_step": records, "visible_gaussians": vis, "parallelism": f"replicas{world}",
                   "programmatic_launch": not args.no_programmatic_launch,
                   "l2": "inputs larger than L2 (params + Adam moments 835 MB, a new 5 MB target per step)"},
        "gpu_launches": forms[chosen]["gpu_launches"],
        "forms": forms,
        "form_switches": {
            "plain_fp32": "reference arithmetic, dense Adam", "graph_fp32": "plain as one CUDA graph per step",
            "culled_fp32": "exact tile culling (images bit-identical to plain)", "culled_graph_fp32": "culled + graph",
            "culled_sparse_fp32": "culled + visibility-masked Adam on the Morton-ordered model + fast blend arithmetic",
            "culled_sparse_graph_fp32": "culled_sparse + graph",
            "precision_bf16_culled_sparse": "culled_sparse + bf16 SH storage and moments + tcgen05 SSIM",
            "precision_bf16_culled_sparse_graph": "precision + graph",
            "precision_bf16_fp32ssim_culled_sparse": "precision with the fp32 CUDA-core SSIM gradient",
            "precision_bf16_fp32ssim_culled_sparse_graph": "precision_bf16_fp32ssim + graph"},
        "chosen_over_plain": round(forms[chosen]["value"] / value, 4),
        "e2e": {"value": forms[chosen]["e2e"], "unit": UNIT, "h2d_bytes_per_step": 1600 * 1064 * 3,
                "d2h_bytes_per_step": 32, "psnr_db_last_step": forms[chosen]["psnr_db_last_step"],
                "pipelining": ("next step's target upload on a copy stream; each step's loss read back "
                               "asynchronously, the host waits for step k - 2 before issuing step k + 1"),
                "results_read": len(e2e_seen), "results_finite": bool(np.all(np.isfinite(e2e_seen)))},
        "reference_cuda": ref_cuda,
        "plain_over_reference_cuda": (round(value / ref_cuda["value"], 4) if ref_cuda and "value" in ref_cuda
                                      else None),
        "chosen_over_reference_cuda": (round(forms[chosen]["value"] / ref_cuda["value"], 4)
                                       if ref_cuda and "value" in ref_cuda else None),
        "e2e_chosen_over_reference_cuda": (round(forms[chosen]["e2e"] / ref_cuda["e2e"], 4)
                                           if ref_cuda and "e2e" in ref_cuda else None),
        "psnr_gate": gate,
        "large_scene": large,
        "roofline": roofline,
        "roofline_plain": roofline_of("plain_fp32"),
        "roofline_dominant": blend_roofline(chosen).get("raster_backward"),
        "roofline_blend": {"chosen": blend_roofline(chosen), "plain": blend_roofline("plain_fp32")},
        "psnr_note": ("psnr_db_last_step is the training view's PSNR after this run's steps from the random "
                      "model; the 0.1 dB condition is checked by psnr_gate: held-out PSNR of plain and chosen "
                      "training runs on the reduced schedule, same scene, density seeds and iterations"),
        "stages": stage_table,
        "stages_culled": {k: round(v, 4) for k, v in culled_stages.items()},
        "stages_culled_sparse": {k: round(v, 4) for k, v in sparse_stages.items()},
        "stages_precision": {k: round(v, 4) for k, v in prec_stages.items()},
        "stages_precision_fp32ssim": {k: round(v, 4) for k, v in prec32_stages.items()},
        "records": {"plain": records, "culled": culled_records},
        "multiview": multiview,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gsn(args)


if __name__ == "__main__":
    main()
