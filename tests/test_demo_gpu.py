"""The OpenCV-free demo programs end to end on a small COLMAP scene: gsn_train
(reference demo/train.cpp) trains from sparse/0/*.bin and PPM images and writes
point_cloud/iteration_N/point_cloud.ply + cfg_args; gsn_render (reference
demo/render.cpp) renders the test views and writes PNG renders / gt /
comparison images and psnr.csv. The PSNR column is recomputed here from the
PLY through the library renderer."""
import os
import subprocess

import numpy as np
import pytest

import colmap_writer as cw
import gsn
import oracle
import scenes

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "gs-native_b200", "bin")


def _write_ring_scene(root, views=16, width=200, height=140, f=180.0, n=15000):
    import torch
    cams = scenes.ring_cameras(views, 6.0, 15.0, width, height, f, f)
    hidden = scenes.random_gaussians(n, 31, mean_sigma=1.2)
    r = gsn.Renderer()
    hp = torch.from_numpy(hidden).cuda()
    img = torch.empty((height, width, 3), device="cuda")
    entries = []
    for k, c in enumerate(cams):
        assert r.render(hp.data_ptr(), n, c, [0, 0, 0], img.data_ptr(), 3) == 0
        rgb = (img * 255).round().clamp(0, 255).to(torch.uint8).cpu().numpy()
        R = np.array(c.R_c_w[:]).reshape(3, 3)
        entries.append({"name": f"view_{k:02d}.jpg", "qvec": cw.matrix_to_quaternion(R),
                        "tvec": np.array(c.t_c_w[:], dtype=np.float64), "image": rgb})
    points, colors = scenes.initial_points(hidden, 3000, 4)
    # COLMAP's principal point is in pixel-edge coordinates: the loader's -0.5
    # shift brings it back to the renderer's pixel-centre convention
    cw.write_scene(str(root), width, height, f, f, cams[0].cx + 0.5, cams[0].cy + 0.5, entries, points,
                   np.clip(np.round(colors * 255), 0, 255))
    return cams


def _run(args):
    p = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return p.stdout


def test_train_and_render_demo(tmp_path):
    scene_dir, out = tmp_path / "scene", tmp_path / "model"
    cams = _write_ring_scene(scene_dir)
    s = gsn.ColmapScene(scene_dir)
    assert len(s.test_cameras) == 2 and len(s.train_cameras) == 14
    # the loaded cameras reproduce the synthetic poses
    byname = {f"view_{k:02d}.jpg": c for k, c in enumerate(cams)}
    for name, cam in zip(s.train_names + s.test_names, s.train_cameras + s.test_cameras):
        ref = byname[name]
        assert np.allclose(cam.R_c_w[:], ref.R_c_w[:], atol=1e-5)
        assert np.allclose([cam.fx, cam.cx, cam.cy], [ref.fx, ref.cx, ref.cy], atol=1e-4)

    log = _run([os.path.join(BIN, "gsn_train"), "--scene", str(scene_dir), "--output", str(out),
                "--iterations", "1200", "--checkpoint", str(tmp_path / "state.ckpt")])
    assert "Training total" in log
    ply = out / "point_cloud" / "iteration_1200" / "point_cloud.ply"
    assert ply.exists() and (out / "cfg_args").read_text().startswith("Namespace(sh_degree=1")
    assert (tmp_path / "state.ckpt").exists()

    render_dir = tmp_path / "renders"
    _run([os.path.join(BIN, "gsn_render"), "--scene", str(scene_dir), "--model", str(ply), "--output",
          str(render_dir), "--split=test"])
    dest = render_dir / "test" / "gs-native"
    rows = (dest / "psnr.csv").read_text().strip().split("\n")
    assert rows[0] == "image,psnr_db" and rows[-1].startswith("mean,")
    psnr = [float(r.split(",")[1]) for r in rows[1:-1]]
    assert len(psnr) == 2 and float(rows[-1].split(",")[1]) == pytest.approx(np.mean(psnr), abs=1e-8)
    assert min(psnr) > 15.0  # held-out views of a 14-view ring after 1,200 updates

    metrics = (dest / "metrics.csv").read_text().strip().split("\n")
    assert metrics[0] == "image,psnr_db,ssim,l1" and len(metrics) == 4

    # recompute from the PLY through the library renderer
    import torch
    st, params = gsn.ply_read(ply)
    assert st == 0
    dp = torch.from_numpy(params).cuda()
    r = gsn.Renderer()
    for k, (cam, target) in enumerate(zip(s.test_cameras, s.test_images)):
        img = torch.empty((cam.height, cam.width, 3), device="cuda")
        assert r.render(dp.data_ptr(), params.shape[1], cam, [0, 0, 0], img.data_ptr(), 3) == 0
        u8 = np.rint(np.clip(img.cpu().numpy(), 0, 1) * np.float32(255)).astype(np.uint8)
        mse = np.mean((u8.astype(np.float64) - target) ** 2) / 255.0 ** 2
        assert -10 * np.log10(mse) == pytest.approx(psnr[k], abs=1e-6)
        fp64 = [float(x) for x in metrics[1 + k].split(",")[1:]]
        want = oracle.eval_metrics(img.cpu().numpy().astype(np.float64), target)
        assert np.allclose(fp64, want[:3], rtol=1e-9, atol=1e-10)
        name = f"{k:05d}.png"
        assert np.array_equal(cw.decode_png(dest / "renders" / name), u8)
        assert np.array_equal(cw.decode_png(dest / "gt" / name), target)
        assert np.array_equal(cw.decode_png(dest / "comparison" / name), np.concatenate([u8, target], axis=1))

    # resuming from the checkpoint continues the schedule
    log = _run([os.path.join(BIN, "gsn_train"), "--scene", str(scene_dir), "--output", str(tmp_path / "resumed"),
                "--iterations", "1500", "--resume", str(tmp_path / "state.ckpt")])
    assert "completed: 1200, single-view updates: 300" in log
    # a non-empty destination is refused, as the reference does
    p = subprocess.run([os.path.join(BIN, "gsn_render"), "--scene", str(scene_dir), "--model", str(ply),
                        "--output", str(render_dir)], capture_output=True, text=True, timeout=600)
    assert p.returncode == 1
