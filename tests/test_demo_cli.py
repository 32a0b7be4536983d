"""Command-line handling of the demo programs (gsn_train, gsn_render) on the
host: the flags each one takes (the reference demos' flags plus the training
forms' switches), and that a bad command line or an unreadable scene ends with
status 1 and a message before any device work; likewise the option checks of the
synthetic full-run driver (synthetic_run.py)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "gs-native_b200", "bin")


def _run(name, *args):
    path = os.path.join(BIN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} is not built (make -C gs-native_b200)")
    return subprocess.run([path, *args], capture_output=True, text=True, timeout=60)


def _flags(help_text):
    return {line.split()[0] for line in help_text.splitlines() if line.strip().startswith("--")}


def test_train_flags():
    out = _run("gsn_train", "--help")
    assert out.returncode == 0
    # reference demo/train.cpp: --scene --output --downscale --iterations
    assert {"--scene", "--output", "--downscale", "--iterations"} <= _flags(out.stdout)
    assert {"--precision", "--graph", "--max_gaussians", "--checkpoint", "--resume", "--culled", "--sparse", "--fast",
            "--fp32_ssim"} <= _flags(out.stdout)


def test_render_flags():
    out = _run("gsn_render", "--help")
    assert out.returncode == 0
    # reference demo/render.cpp: --scene --model --output --downscale --sh_degree --split
    assert {"--scene", "--model", "--output", "--downscale", "--sh_degree", "--split"} <= _flags(out.stdout)


@pytest.mark.parametrize("args", [
    ("--output", "x", "--iterations", "10"),                       # --scene missing
    ("--scene", "x", "--output", "y", "--iterations", "0"),         # no iterations
    ("--scene", "x", "--output", "y", "--no_such_flag"),            # unknown flag
    ("--scene", "x", "--output", "y", "stray"),                     # stray argument
    ("--scene", "x", "--output", "y", "--downscale"),               # value missing
])
def test_train_rejects_bad_command_lines(args):
    out = _run("gsn_train", *args)
    assert out.returncode == 1
    assert "Specify --scene, --output and positive --iterations." in out.stderr


def test_train_reports_an_unreadable_scene(tmp_path):
    out = _run("gsn_train", "--scene", str(tmp_path / "missing"), "--output", str(tmp_path / "out"),
               "--iterations", "10", "--culled", "--sparse", "--fast")
    assert out.returncode == 1
    assert "Reading the COLMAP scene failed." in out.stderr
    assert not (tmp_path / "out").exists()


def test_render_reports_an_unreadable_scene(tmp_path):
    out = _run("gsn_render", "--scene", str(tmp_path / "missing"), "--model", str(tmp_path / "m.ply"),
               "--output", str(tmp_path / "out"))
    assert out.returncode == 1
    assert "failed" in out.stderr


@pytest.mark.parametrize("args", [["--lazy-decay"], ["--lazy-decay", "--sparse", "--graph"]])
def test_synthetic_run_rejects_lazy_decay_outside_eager_sparse_steps(args):
    # lazy moment decay needs the sparse update and eager steps; the driver says
    # so before it touches the device
    import sys
    script = os.path.join(ROOT, "gs-native_b200", "synthetic_run.py")
    out = subprocess.run([sys.executable, script, *args], capture_output=True, text=True, timeout=120)
    assert out.returncode == 2 and "--lazy-decay needs --sparse" in out.stderr
