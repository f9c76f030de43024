"""Checkpoints and the headless frame loop (mpm_run, the counterpart of
Simulation::run): a loaded checkpoint holds the saved state bit for bit and
continues like the saved engine (to 1e-4: slot order changes the order of
float sums); the CLI builds a config's scene, runs frames, writes positions
and checkpoints, and resumes."""
import json
import os
import subprocess

import numpy as np
import pytest

import objgen
from parity import assert_state_close

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "water-sim-cuda_b200", "bin", "mpm_run")


def test_checkpoint_roundtrip(gpu_ok, mpm, tmp_path):
    from mpm_b200 import scenes
    cfg, st, tris = scenes.small_scene(4000, (32, 40, 24), seed=21)
    path = str(tmp_path / "a.ckpt")
    with mpm.Engine(cfg) as e:
        e.init(st)
        e.init_sdf(tris)
        e.step(5)
        e.save_checkpoint(path, note="SIZE_X=32\n")
        saved, sdf = e.get_buffer(), e.get_sdf()
        e.step(5)
        cont = e.get_buffer()
    info = mpm.checkpoint_info(path)
    assert info["n"] == 4000 and info["substeps"] == 5 and info["note"] == "SIZE_X=32\n"
    assert info["config"].size_y == 40 and np.float32(info["config"].dt) == np.float32(cfg.dt)
    with mpm.Engine.load_checkpoint(path) as e:
        assert np.array_equal(e.get_buffer(), saved)
        assert np.array_equal(e.get_sdf(), sdf)
        assert e.stats()["substeps"] == 5
        e.step(5)
        again = e.get_buffer()
    assert_state_close(again, cont.astype(np.float64), saved, rtol=1e-4)


def test_checkpoint_corruption(gpu_ok, mpm, tmp_path):
    from mpm_b200 import scenes
    cfg, st, tris = scenes.small_scene(500, (16, 16, 16), seed=22, obstacle=False)
    path = tmp_path / "b.ckpt"
    with mpm.Engine(cfg) as e:
        e.init(st)
        e.save_checkpoint(str(path))
    raw = bytearray(path.read_bytes())
    raw[200] ^= 0x40
    (tmp_path / "bad.ckpt").write_bytes(bytes(raw))
    (tmp_path / "short.ckpt").write_bytes(bytes(raw[:-10]))
    for name in ("bad.ckpt", "short.ckpt", "none.ckpt"):
        with pytest.raises(mpm.MpmError) as ei:
            mpm.Engine.load_checkpoint(str(tmp_path / name))
        assert ei.value.name == "MPM_ERR_IO"


def _scene_dir(tmp_path, substeps=4):
    (tmp_path / "models").mkdir()
    (tmp_path / "models" / "sphere.obj").write_text(objgen.uv_sphere(1.0, 16, 8))
    (tmp_path / "models" / "torus.obj").write_text(objgen.torus(25.0, 8.0, 24, 12))
    cfg = "\n".join(["SIZE_X=64", "SIZE_Y=64", "SIZE_Z=64", "PADDING=3", "GRAVITY=9.81", "DT=0.01", "GAMMA=-2.0",
                     "COMPRESSION=200.0", "RESOLUTION=1.0", f"SUBSTEPS={substeps}", "SDF_RESOLUTION=64",
                     "WATER=models/sphere.obj;20.0;0.0;5.0;0.0", "OBJECT=models/torus.obj;40.0;0.0;-15.0;0.0"])
    (tmp_path / "config.txt").write_text(cfg + "\n")
    return tmp_path / "config.txt"


def _run(*args):
    r = subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def _positions(path):
    raw = open(path, "rb").read()
    assert raw[:8] == b"MPMPOS01"
    n, frames = np.frombuffer(raw[8:24], np.int64)
    return np.frombuffer(raw[24:], np.float32).reshape(frames, n, 3)


def test_cli_frames_positions_checkpoint_resume(gpu_ok, mpm, tmp_path):
    cfgp = _scene_dir(tmp_path)
    out = _run(cfgp, "--frames", 6, "--positions", tmp_path / "p.bin", "--every", 2, "--checkpoint",
               tmp_path / "c.ckpt", "--quiet")
    assert out["frames"] == 6 and out["substeps_total"] == 24 and out["positions_frames"] == 3
    pos = _positions(tmp_path / "p.bin")
    assert pos.shape == (3, out["particles"], 3) and np.isfinite(pos).all()
    # the same scene through the Python API: identical initial scene
    cfg, st, tris, _ = mpm.build_scene(open(cfgp).read(), str(tmp_path))
    assert st.shape[1] == out["particles"]
    with mpm.Engine(cfg) as e:
        e.init(st)
        e.init_sdf(tris)
        e.step(24)
        ref = e.get_positions()
    assert np.abs(pos[-1] - ref).max() < 1e-3
    info = mpm.checkpoint_info(str(tmp_path / "c.ckpt"))
    assert info["substeps"] == 24 and "WATER=models/sphere.obj" in info["note"]
    (tmp_path / "img").mkdir()
    res = _run("--resume", tmp_path / "c.ckpt", "--frames", 2, "--quiet", "--render", tmp_path / "img",
               "--render-size", "64x48")
    assert res["substeps_total"] == 32 and res["particles"] == out["particles"] and res["rendered_frames"] == 2
    ppm = (tmp_path / "img" / "frame_00002.ppm").read_bytes()
    assert ppm.startswith(b"P6\n64 48\n255\n") and len(ppm) == len(b"P6\n64 48\n255\n") + 64 * 48 * 3


def test_cli_learned_frames(gpu_ok, mpm, tmp_path):
    import mlp_ref
    cfgp = _scene_dir(tmp_path, substeps=8)
    w = mlp_ref.random_params(3)
    mlp_ref.split(w)["W3"][:] *= 0.01
    w.astype("<f4").tofile(tmp_path / "w.bin")
    out = _run(cfgp, "--frames", 3, "--corrector", tmp_path / "w.bin", "--ratio", 4, "--threshold", -1, "--quiet")
    assert out["large_steps"] == 6 and out["fallbacks"] == 0
