"""Precision form: parameter blocks with the 48 SH rows stored as bf16 (10 fp32
geometry rows + 24 float rows of bf16), fp32 blending and accumulation, SH
updates with stochastic rounding. Each stage is checked against the plain FP32
form run on the same parameters with their SH rounded to bf16, so the only
differences left are the ones the precision form introduces on purpose."""
import numpy as np
import pytest

import gsn
import scenes
from helpers import dev, empty, host, sync, torch
from test_density_gpu import random_case

pytestmark = pytest.mark.gpu


def rounded(params):
    """SH rows rounded to bf16 (round to nearest even), as fp32."""
    t = torch()
    out = params.copy()
    out[10:] = t.from_numpy(params[10:]).to(t.bfloat16).float().numpy()
    return out


def bf16_ulp(x):
    e = np.floor(np.log2(np.maximum(np.abs(x), 1e-30)))
    return np.exp2(e - 7)


def scene(n=4096, seed=0):
    params, cam = scenes.single_step_scene()
    if n != params.shape[1]:
        params = scenes.random_gaussians(n, seed)
    tp = scenes.random_gaussians(4096, 1)
    t = torch()
    r = gsn.Renderer()
    tpd = dev(tp)
    img = empty((cam.height, cam.width, 3), t.float32)
    assert r.render(tpd.data_ptr(), 4096, cam, [1, 1, 1], img.data_ptr(), 3) == 0
    target = (img * 255).round().clamp(0, 255).to(t.uint8)
    sync()
    return rounded(params), cam, target


def render_pair(params, cam):
    t = torch()
    n = params.shape[1]
    plain, prec = gsn.Renderer(), gsn.Renderer()
    prec.set_bf16_sh(True)
    p32 = dev(params)
    pb = gsn.to_precision_layout(params, t)
    a = empty((cam.height, cam.width, 3), t.float32)
    b = empty((cam.height, cam.width, 3), t.float32)
    assert plain.render(p32.data_ptr(), n, cam, [1, 1, 1], a.data_ptr(), 3) == 0
    assert prec.render(pb.data_ptr(), n, cam, [1, 1, 1], b.data_ptr(), 3) == 0
    sync()
    return a.cpu().numpy(), b.cpu().numpy()


def test_precision_layout_round_trips():
    t = torch()
    params = scenes.random_gaussians(1001, 4)
    back = gsn.from_precision_layout(gsn.to_precision_layout(params, t), 1001, t).cpu().numpy()
    assert np.array_equal(back[:10], params[:10])
    assert np.array_equal(back[10:], rounded(params)[10:])


def test_render_matches_plain_form_on_bf16_rounded_sh():
    params, cam, _ = scene()
    a, b = render_pair(params, cam)
    # the same arithmetic up to FMA contraction in the SH sum, plus the FP64
    # inversion of near-singular conics
    assert np.max(np.abs(a - b)) <= 1e-5
    assert np.mean(np.abs(a - b) <= 1e-6) > 0.99


def run_steps(params, cam, target, bf16, steps=1, lr=1e-4, tensor_core_loss=False):
    """Steps of either layout. The precision layout switches the solver to the
    tensor-core SSIM; these storage tests keep the fp32 loss kernel so that both
    forms run the same arithmetic and only the bf16 storage differs (the
    tensor-core loss is pinned in test_loss_tc_gpu.py and
    test_precision_error_gpu.py)."""
    t = torch()
    n = params.shape[1]
    r, s = gsn.Renderer(), gsn.Solver()
    r.set_bf16_sh(bf16)
    s.set_bf16_sh(bf16)
    s.set_tensor_core_loss(tensor_core_loss)
    p = gsn.to_precision_layout(params, t) if bf16 else dev(params)
    img = empty((cam.height, cam.width, 3), t.float32)
    for _ in range(steps):
        assert r.render(p.data_ptr(), n, cam, [1, 1, 1], img.data_ptr(), 3) == 0
        assert s.iterate(cam, r, img.data_ptr(), target.data_ptr(), p.data_ptr(), n, lr, 3) == 0
    sync()
    out = gsn.from_precision_layout(p, n, t) if bf16 else p
    m_ptr, v_ptr, _ = s.moments()
    rows = 34 if bf16 else 58
    m = host(m_ptr, np.float32, rows * n)
    if bf16:
        mt = t.from_numpy(m).cuda()
        m = gsn.from_precision_layout(mt, n, t).cpu().numpy()
    else:
        m = m.reshape(58, n)
    return out.cpu().numpy(), m


def test_one_step_matches_plain_form_to_bf16_rounding():
    params, cam, target = scene()
    p32, m32 = run_steps(params, cam, target, False)
    pb, mb = run_steps(params, cam, target, True)
    moved = np.abs(p32 - params)
    # geometry rows: same fp32 arithmetic (backward atomics reorder sums)
    g = slice(0, 10)
    assert np.mean(np.abs(pb[g] - p32[g]) <= 1e-6 + 1e-3 * moved[g]) > 0.999
    # SH rows: the fp32 result, stochastically rounded to one of its bf16 neighbours
    sh = slice(10, 58)
    err = np.abs(pb[sh] - p32[sh])
    assert np.mean(err <= 1.01 * bf16_ulp(p32[sh]) + 1e-7) > 0.999
    errm = np.abs(mb[sh] - m32[sh])
    assert np.mean(errm <= 1.01 * bf16_ulp(m32[sh]) + 1e-12) > 0.999


def test_stochastic_rounding_keeps_small_steps():
    """SH-rest steps (lr 1.25e-4) are below half a bf16 ulp of coefficients
    around 0.05: round-to-nearest would drop them; stochastic rounding must
    move the coefficients like the fp32 form does, on average."""
    params, cam, target = scene()
    steps = 40
    p32, _ = run_steps(params, cam, target, False, steps=steps)
    pb, _ = run_steps(params, cam, target, True, steps=steps)
    rest = [10 + c * 16 + k for c in range(3) for k in range(1, 16)]
    d32 = np.abs(p32[rest] - params[rest]).sum()
    db = np.abs(pb[rest] - params[rest]).sum()
    assert d32 > 0
    assert 0.8 < db / d32 < 1.25, (db, d32)


def test_density_control_copies_bf16_sh_rows_exactly():
    params, s, a = random_case(30_000, 3)
    params = rounded(params)
    n = params.shape[1]
    t = torch()

    def run(bf16):
        ctl = gsn.Density()
        ctl.set_bf16_sh(bf16)
        assert ctl.initialize(n, n) == 0
        sd, ad = dev(s), dev(a)
        for _ in range(2):
            assert ctl.accumulate(sd.data_ptr(), ad.data_ptr(), n) == 0
        rows = 34 if bf16 else 58
        src = gsn.device_alloc(rows * 4 * n)
        block = gsn.to_precision_layout(params, t) if bf16 else dev(params)
        gsn.memcpy(src, block.data_ptr(), rows * 4 * n)
        st, p, m, ch = ctl.control(src, n, 3.0, 0.0002, 0.01, 0.005, 20.0, 7, 0.0008)
        assert st == 0
        sync()
        out = np.zeros((rows * m,), np.float32)
        gsn.memcpy(out.ctypes.data, p, out.nbytes)
        gsn.device_free(p)
        if bf16:
            return gsn.from_precision_layout(t.from_numpy(out).cuda(), m, t).cpu().numpy(), m, ch
        return out.reshape(58, m), m, ch

    ref, m32, ch32 = run(False)
    mine, mb, chb = run(True)
    assert m32 == mb and ch32 == chb and m32 != n
    assert np.array_equal(ref.view(np.uint32), mine.view(np.uint32))


def test_trainer_precision_form_trains_like_plain_form():
    cams = scenes.ring_cameras(12, 6.0, 15.0, 240, 160, 210.0, 210.0)
    hidden = scenes.random_gaussians(20000, 21, mean_sigma=1.2)
    t = torch()
    r = gsn.Renderer()
    hp = dev(hidden)
    img = empty((160, 240, 3), t.float32)
    images = []
    for c in cams:
        assert r.render(hp.data_ptr(), hidden.shape[1], c, [0, 0, 0], img.data_ptr(), 3) == 0
        images.append((img * 255).round().clamp(0, 255).to(t.uint8).cpu().numpy())
    points, colors = scenes.initial_points(hidden, 5000, 2)
    train_c, train_i = cams[1:], images[1:]
    # Three runs per form, compared on their medians. Runs differ only through
    # the order of the backward's float atomics, which the density decisions of
    # this small 1,500-iteration scene amplify: over 8 fresh runs each, plain
    # ended at 19.0-19.5 dB and the precision form (bf16 SH storage with
    # stochastic rounding) at 18.5-19.6 dB, with single runs in the test suite
    # as low as 17.5 dB. The full-scale held-out gate in bench.py measures the
    # forms' quality; this test checks that training is not systematically off.
    result = {}
    for precision in (0, 1):
        runs = []
        for _ in range(3):
            opts = gsn.TrainingOptions.defaults(densify_from=100, densify_until=600, densify_interval=100,
                                                opacity_reset_interval=100000, precision=precision)
            tr = gsn.Trainer()
            assert tr.initialize(train_c, train_i, points, colors, opts) == 0
            before, _ = tr.evaluate(cams[:1], images[:1])
            assert tr.train(1500) == 0
            after, _ = tr.evaluate(cams[:1], images[:1])
            runs.append((before, after, tr.state()["count"]))
            tr.close()
        result[precision] = (runs[0][0], float(np.median([r[1] for r in runs])), runs)
    assert result[0][1] > result[0][0] + 3.0
    assert result[1][1] > result[1][0] + 3.0
    assert abs(result[1][1] - result[0][1]) < 0.5, result

