"""The FluidGPU driver executable (the reference's main.cpp over the C ABI).

CPU: the executable is built beside the library, prints its usage and fails
cleanly (exit 1, a message) on a missing config.  GPU: on a small scene given
by a reference-format label file and config.json, the driver's frames, initial
particles, body surface points and csvRes.csv match the same run made through
the ctypes binding (fp_config_load_json, fp_load_labels, fp_load_sdf,
fp_seed_particles, fp_save_ply, fp_run).
"""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_l2

DRIVER = os.path.join(ROOT, "fluidprjct_b200", "_lib", "FluidGPU")


def test_driver_usage_and_missing_config(tmp_path):
    assert os.access(DRIVER, os.X_OK), "FluidGPU is built by fluidprjct_b200/build.py"
    r = subprocess.run([DRIVER, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "usage: FluidGPU" in r.stderr
    r = subprocess.run([DRIVER, str(tmp_path / "missing.json")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "cannot open config" in r.stderr
    r = subprocess.run([DRIVER, "a", "b"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1


def _write_scene(tmp, body):
    from fluidprjct_b200 import scenes
    n = 24
    lab = scenes.box_3d(n, n, n, 1.0 / n, 0.5, 0.6, 1.0)
    scenes.write_labels3d(str(tmp / "labels.txt"), lab)
    cfg = {"dt": 0.004, "dx": 1.0 / n, "PIC_WEIGHT": 0.05, "iterPerFrame": 2, "outputFormat": "PLY",
           "inputLabelData": str(tmp / "labels.txt"), "frameAmount": 3,
           "outputTemplate": str(tmp / "out" / "particles_"), "activeBody": bool(body),
           "body_x": 0.7, "body_y": 0.5, "body_z": 0.5, "body_mass": 1.0, "body_radius": 0.12 if body else 0.0,
           "body_density": 0.5, "ppc": 4, "seed": 7, "solver": "pcg_mg", "advection": "rk2",
           "collision": "sdf" if body else "labels", "initialParticles": str(tmp / "out" / "particles_-1.ply")}
    os.makedirs(tmp / "out", exist_ok=True)
    with open(tmp / "config.json", "w") as f:
        json.dump(cfg, f)
    return cfg


@pytest.mark.gpu
@pytest.mark.parametrize("body", [False, True])
def test_driver_matches_the_same_run_through_ctypes(tmp_path, body):
    import ctypes as C
    from fluidprjct_b200 import capi
    drv = tmp_path / "driver"
    py = tmp_path / "ctypes"
    for d in (drv, py):
        os.makedirs(d)
        _write_scene(d, body)
    r = subprocess.run([DRIVER, str(drv / "config.json")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Number of particles is" in r.stdout and "fps = " in r.stdout

    cfg = capi.default_config()
    lab = C.create_string_buffer(1024)
    frames = C.c_int(100)
    assert capi.lib().fp_config_load_json(str(py / "config.json").encode(), C.byref(cfg), lab, 1024,
                                          C.byref(frames)) == 0
    s = capi.Solver(cfg)
    s.load_labels(lab.value.decode())
    if body:
        s.load_sdf(None)
    s.seed_particles(cfg.ppc, cfg.seed)
    s.save_ply(str(py / "out" / "particles_-1.ply"))
    s.run(frames.value)
    s.close()

    names = sorted(os.listdir(drv / "out"))
    assert names == sorted(os.listdir(py / "out"))
    frame_files = [f"particles_{i}.ply" for i in range(frames.value + 1)]
    assert set(frame_files + ["particles_-1.ply"]) <= set(names)
    if body:
        assert "csvRes.csv" in names and "body_0.ply" in names
    for f in names:
        a, b = drv / "out" / f, py / "out" / f
        if f.endswith(".ply"):
            pa, _ = capi.read_ply_file(str(a))
            pb, _ = capi.read_ply_file(str(b))
            assert pa.shape == pb.shape
            # the same step twice; P2G's shared-memory sums are order-dependent in the last bits
            assert rel_l2(pa, pb) <= 1e-5, f
        else:
            ca = np.loadtxt(a, delimiter=",", skiprows=1)
            cb = np.loadtxt(b, delimiter=",", skiprows=1)
            assert ca.shape == cb.shape and np.allclose(ca, cb, atol=1e-5), f
