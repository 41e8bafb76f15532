"""The C ABI without a GPU: symbols, defaults, host-side parsers, scenes."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, reference_file

HEADER = os.path.join(ROOT, "include", "fluidprjct.h")


def header_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from fluidprjct_b200 import capi
    lib = capi.lib()
    syms = header_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # and the binding declares a signature for each of them
    assert sorted(capi.declared_symbols()) == syms
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (fp_\w+)", out))
    assert set(syms) <= exported


C_CALLER = r"""
#include <stdio.h>
#include <string.h>
#include "fluidprjct.h"
int main(int argc, char** argv) {
    fp_config c;
    char labels[64];
    int frames = 0;
    float pos[6] = {0.1f, 0.2f, 0.3f, 0.4f, 0.5f, 0.6f}, back[6] = {0};
    int64_t n = 2;
    int has_vel = -1;
    fp_solver* s = NULL;
    if (argc < 3) return 2;
    fp_config_default(&c);
    printf("default %d %d %g\n", c.dim, c.ppc, (double)c.pic_weight);
    if (fp_config_load_json(argv[1], &c, labels, sizeof labels, &frames) != FP_OK) return 3;
    printf("json %g %d %s %s\n", (double)c.dt, frames, labels, c.output_template);
    c.dim = 5;
    printf("create %d %d\n", fp_create(&c, &s), s == NULL);
    if (fp_write_particle_file(argv[2], pos, NULL, n, FP_OUT_PLY_BINARY) != FP_OK) return 4;
    if (fp_read_ply_file(argv[2], &n, back, NULL, &has_vel) != FP_OK) return 5;
    printf("ply %lld %d %d\n", (long long)n, has_vel, memcmp(pos, back, sizeof pos) == 0);
    return 0;
}
"""


def test_header_is_plain_c(tmp_path):
    """The ABI is what a cgo / FFI binding would compile: a C99 caller built
    with gcc -pedantic against include/fluidprjct.h links the library and
    calls its host-side entry points (no GPU work)."""
    import shutil
    from fluidprjct_b200 import capi
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no gcc")
    src = tmp_path / "caller.c"
    src.write_text(C_CALLER)
    exe = tmp_path / "caller"
    libdir = os.path.dirname(capi.LIB_PATH)
    r = subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                        str(src), "-L", libdir, "-lfluidprjct_b200", "-Wl,-rpath," + libdir, "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    cfg = tmp_path / "config.json"
    cfg.write_text('{"dt": 0.005, "frameAmount": 12, "inputLabelData": "InputData/labels.txt",'
                   ' "outputTemplate": "OutputData/particles_"}')
    r = subprocess.run([str(exe), str(cfg), str(tmp_path / "p.ply")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, (r.stdout, r.stderr)
    assert r.stdout.splitlines() == ["default 3 4 0.01", "json 0.005 12 InputData/labels.txt OutputData/particles_",
                                     "create %d 1" % capi.FP_ERR_ARG, "ply 2 1 1"]  # binary PLY carries vel


def test_config_defaults_match_reference():
    from fluidprjct_b200 import capi
    c = capi.default_config()
    # main.cpp:18-48 and FluidSolver3D.cuh:71, FluidSolver3D.cu:3092
    assert (c.dim, c.iter_per_frame, c.ppc) == (3, 1, 4)
    f32 = lambda x: float(np.float32(x))
    assert (c.dt, c.dx, c.pic_weight, c.cfl, c.body_mass) == (f32(0.02), f32(0.1), f32(0.01), f32(0.1), 50.0)
    assert list(c.body_pos) == pytest.approx([0.5, 0.5, 0.5])
    assert c.output_template == b"InputData/particles_"
    assert c.solver == capi.SOLVER_PCG and c.advection == capi.ADVECT_RK3REF
    assert c.scheme == capi.SCHEME_DEFAULT
    # additions: MG warm start on, the finest level's sweep pairs at their default
    assert (c.warm_start, c.mg_sweeps) == (1, 0)
    # the ctypes mirrors have the C sizes (int64 + int32 x 2 appended to the stats)
    assert C.sizeof(capi.FpStepStats) % 8 == 0
    # a misspelt field is an error, not a silently ignored attribute
    with pytest.raises(TypeError, match="pic_wieght"):
        capi.default_config(pic_wieght=0.1)
    c = capi.default_config(pic_weight=0.25, body_pos=(0.1, 0.2, 0.3), solver="pcg_mg", output_template="o/p_")
    assert c.pic_weight == 0.25 and list(c.body_pos) == pytest.approx([0.1, 0.2, 0.3])
    assert c.solver == capi.SOLVER_PCG_MG and c.output_template == b"o/p_"


def test_create_rejects_bad_schemes():
    """fp_create checks the configuration before touching the GPU."""
    from fluidprjct_b200 import capi
    for kw in ({"dim": 3, "scheme": capi.SCHEME_REF2D}, {"dim": 2, "scheme": 7}):
        cfg = capi.default_config(**kw)
        h = C.c_void_p()
        assert capi.lib().fp_create(C.byref(cfg), C.byref(h)) == capi.FP_ERR_ARG and not h.value


def test_config_json(tmp_path):
    from fluidprjct_b200 import capi
    p = tmp_path / "config.json"
    # the keys of the reference's InputData/config.json:1-14 plus additions
    p.write_text('{"dt": 0.005, "dx": 0.02, "PIC_WEIGHT": 0.001, "iterPerFrame": 1, "outputFormat": "PLY",\n'
                 ' "inputLabelData": "InputData/labels_gaussian.txt", "frameAmount": 280,\n'
                 ' "outputTemplate": "OutputData/particles_", "body_x": 0.5, "body_y": 0.2, "body_z": 0.5,\n'
                 ' "body_mass": 0.03, "activeBody": true, "solver": "pcg_mixed", "advection": "rk2",'
                 ' "seed": 7, "mg_sweeps": 3, "warm_start": 0, "nested": {"a": [1, 2, {"b": null}]}}')
    cfg = capi.default_config()
    lab = C.create_string_buffer(256)
    frames = C.c_int(0)
    rc = capi.lib().fp_config_load_json(str(p).encode(), C.byref(cfg), lab, 256, C.byref(frames))
    assert rc == capi.FP_OK
    f32 = lambda x: float(np.float32(x))
    assert (cfg.dt, cfg.dx, cfg.pic_weight, cfg.body_mass) == (f32(0.005), f32(0.02), f32(0.001), f32(0.03))
    assert cfg.active_body == 1
    assert list(cfg.body_pos) == pytest.approx([0.5, 0.2, 0.5])
    assert cfg.output_template == b"OutputData/particles_" and cfg.output_format == capi.OUT_PLY
    assert lab.value == b"InputData/labels_gaussian.txt" and frames.value == 280
    assert cfg.solver == capi.SOLVER_PCG_MIXED and cfg.advection == capi.ADVECT_RK2 and cfg.seed == 7
    assert (cfg.mg_sweeps, cfg.warm_start) == (3, 0)
    bad = tmp_path / "bad.json"
    bad.write_text('{"dt": 0.1, "solver": "magic"}')
    assert capi.lib().fp_config_load_json(str(bad).encode(), C.byref(cfg), None, 0, None) == capi.FP_ERR_IO


def test_reference_class_knobs_map_to_the_config():
    """FluidSolver3D keeps the reference class's public knobs and defaults
    (FluidSolver3D.cuh:156-166: PIC_WEIGHT 0.5, iterPerFrame 10, outputFormat
    PLY, outputTemplate "InputData/particles_", four particles per cell at
    :71) and forwards them, and its additions, to fp_config."""
    from fluidprjct_b200 import capi
    from fluidprjct_b200.solver import FluidSolver3D
    f = FluidSolver3D(5, 5, 5, 0.02, 0.005)
    c = f._config()
    f32 = lambda x: float(np.float32(x))
    assert (c.dx, c.dt, c.pic_weight, c.iter_per_frame, c.ppc) == (f32(0.02), f32(0.005), 0.5, 10, 4)
    assert c.output_format == capi.OUT_PLY and c.output_template == b"InputData/particles_"
    assert c.active_body == 0 and c.dim == 3
    f.PIC_WEIGHT, f.iterPerFrame, f.outputTemplate = 0.001, 1, "OutputData/particles_"
    f.activeBody, f.initialBodyPos, f.bodyMass = True, (0.5, 0.2, 0.5), 0.03
    for fmt, want in (("PLY", capi.OUT_PLY), ("OFF", capi.OUT_OFF), ("PLY_BINARY", capi.OUT_PLY_BINARY),
                      ("NONE", capi.OUT_NONE), ("OBJ", capi.OUT_OFF)):
        f.outputFormat = fmt
        assert f._config().output_format == want, fmt
    c = f._config()
    assert (c.pic_weight, c.iter_per_frame, c.active_body) == (f32(0.001), 1, 1)
    assert c.output_template == b"OutputData/particles_" and c.body_mass == f32(0.03)
    assert list(c.body_pos) == pytest.approx([0.5, 0.2, 0.5])
    g = FluidSolver3D(dx=0.1, dt=0.02, solver="pcg_mg", advection="rk2", seed=9)
    c = g._config()
    assert (c.solver, c.advection, c.seed) == (capi.SOLVER_PCG_MG, capi.ADVECT_RK2, 9)
    with pytest.raises(TypeError):
        FluidSolver3D(dx=0.1, dt=0.02, sovler="pcg_mg")._config()


def _load_json(path, label_len=256):
    from fluidprjct_b200 import capi
    cfg = capi.default_config()
    lab = C.create_string_buffer(label_len) if label_len else None
    frames = C.c_int(-1)
    rc = capi.lib().fp_config_load_json(str(path).encode(), C.byref(cfg), lab, label_len, C.byref(frames))
    return rc, cfg, lab, frames.value


def test_config_json_strings_and_formats(tmp_path):
    """String escapes decode as jsoncpp decodes them (RFC 8259: \\" \\\\ \\/ \\b
    \\f \\n \\r \\t and \\uXXXX with surrogate pairs, to UTF-8); outputFormat
    maps "PLY" to PLY and anything else to OFF as main.cpp:25-31 does, plus this
    library's PLY_BINARY and NONE; the label path is cut to the caller's
    buffer."""
    from fluidprjct_b200 import capi
    p = tmp_path / "esc.json"
    p.write_text('{"outputTemplate": "Out\\/d\\\\x\\"q\\tz\\u00e9\\ud83d\\ude00\\b\\f\\r\\n",'
                 ' "inputLabelData": "InputData/labels_gaussian.txt", "outputFormat": "PLY_BINARY"}')
    rc, cfg, lab, _ = _load_json(p)
    assert rc == capi.FP_OK
    assert cfg.output_template == 'Out/d\\x"q\tzé\U0001F600\b\f\r\n'.encode("utf-8")
    assert cfg.output_format == capi.OUT_PLY_BINARY
    rc, _, lab, _ = _load_json(p, label_len=10)
    assert rc == capi.FP_OK and lab.value == b"InputData"
    for fmt, want in (("PLY", capi.OUT_PLY), ("NONE", capi.OUT_NONE), ("OBJ", capi.OUT_OFF), ("ply", capi.OUT_OFF)):
        p.write_text('{"outputFormat": "%s"}' % fmt)
        rc, cfg, _, _ = _load_json(p)
        assert rc == capi.FP_OK and cfg.output_format == want, fmt


def test_config_json_rejects_malformed_input(tmp_path):
    """Missing files, malformed JSON, bad escapes, lone surrogates and unknown
    enumerated values are FP_ERR_IO.  A numeric key holding another type is
    ignored and keeps its default (where jsoncpp's asFloat() would throw), and
    nested values of any kind are skipped."""
    from fluidprjct_b200 import capi
    assert _load_json(tmp_path / "missing.json")[0] == capi.FP_ERR_IO
    p = tmp_path / "c.json"
    for text in ('{"dt": 0.1', '{"dt" 0.1}', '[1, 2]', '{"dt": }', '{"dt": 0.1,, "dx": 1}',
                 '{"outputTemplate": "a\\qb"}', '{"outputTemplate": "\\ud83d"}', '{"outputTemplate": "\\ude00"}',
                 '{"outputTemplate": "\\u12"}', '{"outputTemplate": "abc}',
                 '{"collision": "mesh"}', '{"advection": "euler"}', '{"solver": "cg"}'):
        p.write_text(text)
        assert _load_json(p)[0] == capi.FP_ERR_IO, text
    p.write_text('{"dt": "fast", "dx": 0.25, "nested": {"k": [true, false, null, "s", {"x": -1e-3}]}}')
    rc, cfg, _, _ = _load_json(p)
    d = capi.default_config()
    assert rc == capi.FP_OK and cfg.dt == d.dt and cfg.dx == 0.25


@pytest.mark.parametrize("name,dim", [("labels_simple3d", 3), ("labels_3d_sphere", 3), ("labels_bathymetry", 3),
                                      ("labels_simple", 2), ("labels_colimn", 2)])
def test_host_label_reader(golden_labels, name, dim, tmp_path):
    from fluidprjct_b200 import capi, scenes
    exp = golden_labels[name]
    path = reference_file("InputData", name + ".txt")
    if path is None:
        path = str(tmp_path / "l.txt")
        (scenes.write_labels3d if dim == 3 else scenes.write_labels2d)(path, exp)
    assert np.array_equal(capi.read_label_file(path, dim), exp)


def test_label_reader_rejects_corrupt_files(tmp_path):
    from fluidprjct_b200 import capi
    p = tmp_path / "bad.txt"
    p.write_text("3 3 1\nSSS\nSXS\nSSS\n")
    with pytest.raises(capi.FluidError):
        capi.read_label_file(p, 3)
    p.write_text("3 3 2\nSSS\nSFS\nSSS\n")  # truncated
    with pytest.raises(capi.FluidError):
        capi.read_label_file(p, 3)
    with pytest.raises(capi.FluidError):
        capi.read_label_file(tmp_path / "missing.txt", 3)


def test_ply_reader_ascii_and_binary(golden_particles, tmp_path):
    from fluidprjct_b200 import capi
    pos = golden_particles
    # ascii, positions only (the reference's writer, utility.cu:91-109)
    a = tmp_path / "a.ply"
    with open(a, "w") as f:
        f.write(f"ply\nformat ascii 1.0\nelement vertex {len(pos)}\nproperty float x\nproperty float y\n"
                "property float z\nend_header\n")
        np.savetxt(f, pos, fmt="%.9g")
    p2, v2 = capi.read_ply_file(a)
    assert v2 is None and np.array_equal(p2, pos)
    ref_ply = reference_file("InputData", "particles_-1.ply")
    if ref_ply:
        p3, _ = capi.read_ply_file(ref_ply)
        assert np.array_equal(p3, pos)
    # binary little endian with velocities and an extra double property
    rng = np.random.default_rng(1)
    vel = rng.standard_normal(pos.shape).astype(np.float32)
    b = tmp_path / "b.ply"
    rec = np.zeros(len(pos), dtype=[("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("q", "<f8"), ("vx", "<f4"),
                                    ("vy", "<f4"), ("vz", "<f4")])
    rec["x"], rec["y"], rec["z"] = pos.T
    rec["vx"], rec["vy"], rec["vz"] = vel.T
    with open(b, "wb") as f:
        f.write((f"ply\nformat binary_little_endian 1.0\nelement vertex {len(pos)}\nproperty float x\n"
                 "property float y\nproperty float z\nproperty double q\nproperty float vx\nproperty float vy\n"
                 "property float vz\nend_header\n").encode())
        f.write(rec.tobytes())
    p4, v4 = capi.read_ply_file(b)
    assert np.array_equal(p4, pos) and np.array_equal(v4, vel)
    # truncated files fail loudly
    t = tmp_path / "t.ply"
    t.write_bytes(open(b, "rb").read()[:-10])
    with pytest.raises(capi.FluidError):
        capi.read_ply_file(t)


def test_scene_cell_counts():
    from fluidprjct_b200 import scenes
    lab = scenes.dam_break_3d(128)
    assert int((lab == 1).sum()) == 50 * 76 * 126 == 478800   # x<0.4, y<0.6, z<1 inside the walls
    lab2 = scenes.dam_break_2d(64)
    assert int((lab2 == 1).sum()) == 25 * 31 == 775
    pool = scenes.pool_3d(160)
    assert int((pool == 1).sum()) == 158 * 55 * 158
    assert (lab[0] == 0).all() and (lab[:, -1] == 0).all() and (lab[:, :, 0] == 0).all()


def test_scene_file_round_trip(tmp_path):
    from fluidprjct_b200 import capi, scenes
    lab = scenes.random_boxes(5, n=20)
    p = tmp_path / "s.txt"
    scenes.write_labels3d(p, lab)
    assert np.array_equal(capi.read_label_file(p, 3), lab)


def test_particle_writer_formats(tmp_path):
    """ASCII PLY / OFF lines are "x y z" as an ostream of floats prints them
    (save3dParticlesToPLY / save3dParticlesToOFF, utility.cu:91-127): %g with six significant digits.
    Binary PLY round-trips exactly through the reader."""
    from fluidprjct_b200 import capi
    rng = np.random.default_rng(0)
    odd = [0.0, -0.0, 1e-5, 1.23456789e-5, 1e-4, 123456.7, 1234567.0, 1e-30, -7.5e20, 0.5, 1 / 3, 2 / 3, 3.4e38,
           -2.0 ** -126, 9.999995, 99999.95]
    pos = np.concatenate([rng.uniform(-2, 2, 3 * 300_000), odd, [0.25, 0.5]]).astype(np.float32).reshape(-1, 3)
    vel = rng.uniform(-1, 1, pos.shape).astype(np.float32)
    lib = capi.lib()
    p = tmp_path / "a.ply"
    assert lib.fp_write_particle_file(str(p).encode(), capi.ptr(pos), None, len(pos), capi.OUT_PLY) == 0
    lines = p.read_bytes().decode().split("\n")
    assert lines[:6] == ["ply", "format ascii 1.0", f"element vertex {len(pos)}", "property float x",
                         "property float y", "property float z"] and lines[6] == "end_header"
    body = lines[7:-1]
    assert len(body) == len(pos)
    idx = list(range(0, len(pos), 997)) + list(range(len(pos) - 8, len(pos)))
    for q in idx:
        assert body[q] == "%g %g %g" % tuple(float(v) for v in pos[q]), q
    o = tmp_path / "a.off"
    assert lib.fp_write_particle_file(str(o).encode(), capi.ptr(pos), None, len(pos), capi.OUT_OFF) == 0
    assert o.read_text().split("\n")[:2] == ["OFF", f"{len(pos)} 0 0"]
    b = tmp_path / "b.ply"
    assert lib.fp_write_particle_file(str(b).encode(), capi.ptr(pos), capi.ptr(vel), len(pos),
                                      capi.OUT_PLY_BINARY) == 0
    n = C.c_int64()
    hv = C.c_int()
    lib.fp_read_ply_file(str(b).encode(), C.byref(n), None, None, C.byref(hv))
    p2, v2 = np.zeros_like(pos), np.zeros_like(vel)
    lib.fp_read_ply_file(str(b).encode(), C.byref(n), capi.ptr(p2), capi.ptr(v2), C.byref(hv))
    assert n.value == len(pos) and hv.value == 1 and np.array_equal(p2, pos) and np.array_equal(v2, vel)
