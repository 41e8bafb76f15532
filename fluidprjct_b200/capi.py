"""ctypes binding of the C ABI declared in ``include/fluidprjct.h``.

The native library is required: importing this module on a machine without the
built ``_lib/libfluidprjct_b200.so`` raises, and there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# FLUIDPRJCT_LIB may name another build of the same library (for example one
# built with different tuning macros); by default the in-tree build is used.
LIB_PATH = os.environ.get("FLUIDPRJCT_LIB") or os.path.join(HERE, "_lib", "libfluidprjct_b200.so")

FP_OK, FP_ERR_ARG, FP_ERR_IO, FP_ERR_CUDA, FP_ERR_STATE, FP_ERR_NO_FLUID, FP_ERR_SOLVER, FP_ERR_TIMEOUT = (
    0, -1, -2, -3, -4, -5, -6, -7)
SOLID, FLUID, AIR, BODY = 0, 1, 2, 3
OUT_PLY, OUT_OFF, OUT_PLY_BINARY, OUT_NONE = 0, 1, 2, 3
SOLVER_PCG, SOLVER_PCG_MIXED, SOLVER_PCG_MG, SOLVER_PCG_LEARNED, SOLVER_PCG_LEARNED_MIXED = 0, 1, 2, 3, 4
ADVECT_RK3REF, ADVECT_RK2 = 0, 1
SCHEME_DEFAULT, SCHEME_REF2D = 0, 1
BODY_FORCES_FACE_FRACTION, BODY_FORCES_REFERENCE = 0, 1
COLLISION_LABELS, COLLISION_SDF = 0, 1
GRID_U, GRID_V, GRID_W, GRID_U_SAVED, GRID_V_SAVED, GRID_W_SAVED, GRID_P, GRID_RHS = range(8)
(PHASE_LABEL, PHASE_P2G, PHASE_SAVE, PHASE_FORCES, PHASE_PRESSURE, PHASE_PROJECT, PHASE_BODY, PHASE_G2P,
 PHASE_ADVECT, PHASE_CLEANUP) = range(10)

SOLVER_NAMES = {"pcg": SOLVER_PCG, "pcg_mixed": SOLVER_PCG_MIXED, "pcg_mg": SOLVER_PCG_MG,
                "pcg_learned": SOLVER_PCG_LEARNED, "pcg_learned_mixed": SOLVER_PCG_LEARNED_MIXED}


class FpConfig(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("dx", C.c_float), ("dt", C.c_float), ("pic_weight", C.c_float),
        ("iter_per_frame", C.c_int), ("output_format", C.c_int), ("output_template", C.c_char * 256),
        ("active_body", C.c_int), ("body_pos", C.c_float * 3), ("body_mass", C.c_float),
        ("ppc", C.c_int), ("seed", C.c_uint32), ("solver", C.c_int), ("advection", C.c_int), ("cfl", C.c_float),
        ("tol", C.c_double), ("max_iters", C.c_int), ("body_radius", C.c_float), ("body_density", C.c_float),
        ("device", C.c_int), ("scheme", C.c_int), ("extrapolate", C.c_int), ("body_forces", C.c_int),
        ("mg_sweeps", C.c_int),
        ("warm_start", C.c_int),
        ("collision", C.c_int),
        ("body_sdf", C.c_char * 256),
    ]


class FpStepStats(C.Structure):
    _fields_ = [
        ("step", C.c_int64), ("num_particles", C.c_int64), ("num_fluid_cells", C.c_int32), ("pcg_iters", C.c_int32),
        ("outer_iters", C.c_int32), ("fallback", C.c_int32), ("solve_status", C.c_int32), ("pad_", C.c_int32),
        ("residual", C.c_double),
        ("t_label", C.c_float), ("t_p2g", C.c_float), ("t_forces", C.c_float), ("t_pressure", C.c_float),
        ("t_project", C.c_float), ("t_body", C.c_float), ("t_g2p", C.c_float), ("t_advect", C.c_float),
        ("t_total", C.c_float), ("guess_relres", C.c_float),
        ("body_pos", C.c_double * 3), ("body_vel", C.c_double * 3), ("body_omega", C.c_double * 3),
        ("body_angles", C.c_double * 3), ("body_force", C.c_double * 3), ("body_torque", C.c_double * 3),
        ("kernel_launches", C.c_int64), ("t_pcg", C.c_float), ("t_learned", C.c_float),
        ("particles_removed", C.c_int64), ("advect_capped", C.c_int32), ("pad2_", C.c_int32),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            if name.startswith("pad"):
                continue
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class FluidError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} (status {code})")
        self.code = code


_lib = None

# Every symbol the header declares, with (restype, argtypes).
_P = C.c_void_p
_SIGS = {
    "fp_config_default": (C.c_int, [_P]),
    "fp_config_load_json": (C.c_int, [C.c_char_p, _P, C.c_char_p, C.c_size_t, _P]),
    "fp_create": (C.c_int, [_P, _P]),
    "fp_destroy": (C.c_int, [_P]),
    "fp_last_error": (C.c_char_p, [_P]),
    "fp_load_labels": (C.c_int, [_P, C.c_char_p]),
    "fp_set_labels": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int]),
    "fp_get_dims": (C.c_int, [_P, _P, _P, _P]),
    "fp_load_sdf": (C.c_int, [_P, C.c_char_p]),
    "fp_set_paddle": (C.c_int, [_P, C.c_float, C.c_float, C.c_float]),
    "fp_set_labels_from_levelsets": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int]),
    "fp_read_levelset_file": (C.c_int, [C.c_char_p, _P, _P]),
    "fp_write_particle_file": (C.c_int, [C.c_char_p, _P, _P, C.c_int64, C.c_int]),
    "fp_scene_seabed": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_uint32,
                                  C.c_float]),
    "fp_seed_particles": (C.c_int, [_P, C.c_int, C.c_uint32]),
    "fp_set_particles": (C.c_int, [_P, _P, _P, C.c_int64]),
    "fp_load_ply": (C.c_int, [_P, C.c_char_p]),
    "fp_save_ply": (C.c_int, [_P, C.c_char_p, C.c_int]),
    "fp_num_particles": (C.c_int64, [_P]),
    "fp_get_particles": (C.c_int, [_P, _P, _P, C.c_int64]),
    "fp_step": (C.c_int, [_P, C.c_int]),
    "fp_run": (C.c_int, [_P, C.c_int]),
    "fp_run_phase": (C.c_int, [_P, C.c_int]),
    "fp_get_grid": (C.c_int, [_P, C.c_int, _P, C.c_int64]),
    "fp_set_grid": (C.c_int, [_P, C.c_int, _P, C.c_int64]),
    "fp_get_labels": (C.c_int, [_P, _P, C.c_int64]),
    "fp_get_grid_device": (C.c_int, [_P, C.c_int, _P, C.c_int64]),
    "fp_get_labels_device": (C.c_int, [_P, _P, C.c_int64]),
    "fp_load_learned": (C.c_int, [_P, C.c_char_p]),
    "fp_unet_num_params": (C.c_int64, []),
    "fp_unet_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, _P]),
    "fp_unet_destroy": (None, [_P]),
    "fp_unet_last_error": (C.c_char_p, [_P]),
    "fp_unet_cuda_stream": (C.c_void_p, [_P]),
    "fp_unet_get_params": (C.c_int, [_P, _P, C.c_int64]),
    "fp_unet_set_params": (C.c_int, [_P, _P, C.c_int64]),
    "fp_unet_save": (C.c_int, [_P, C.c_char_p]),
    "fp_unet_load": (C.c_int, [_P, C.c_char_p]),
    "fp_unet_forward": (C.c_int, [_P, _P, _P, _P]),
    "fp_unet_loss_grad": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "fp_unet_train_step": (C.c_int, [_P, _P, _P, _P, C.c_float, _P]),
    "fp_set_body_state": (C.c_int, [_P, _P, _P, _P]),
    "fp_stats": (C.c_int, [_P, _P]),
    "fp_cuda_stream": (C.c_void_p, [_P]),
    "fp_set_wait_limit": (C.c_int, [_P, C.c_int64]),
    "fp_set_step_log": (C.c_int, [_P, C.c_char_p]),
    "fp_save_state": (C.c_int, [_P, C.c_char_p]),
    "fp_load_state": (C.c_int, [_P, C.c_char_p]),
    "fp_pressure_solve": (C.c_int, [_P, _P, _P, C.c_int64, _P, _P]),
    "fp_solve_csr_upper": (C.c_int, [C.c_int, _P, _P, _P, _P, _P, C.c_double, C.c_int, _P, _P]),
    "fp_solve_csr_upper_noalloc": (C.c_int, [C.c_int, _P, _P, _P, _P, _P, C.c_double, C.c_int, _P, _P, _P]),
    "fp_read_label_file": (C.c_int, [C.c_char_p, C.c_int, _P, _P]),
    "fp_read_ply_file": (C.c_int, [C.c_char_p, _P, _P, _P, _P]),
    "fp_version": (C.c_char_p, []),
}


def lib():
    """Load the native library (it must have been built; no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"native library missing: {LIB_PATH}; run `python fluidprjct_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    return list(_SIGS)


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def read_levelset_file(path) -> np.ndarray:
    """A 2D level-set file of the reference's DistrGen tools as an (H, W) array."""
    dims = np.zeros(2, np.int32)
    rc = lib().fp_read_levelset_file(str(path).encode(), ptr(dims), None)
    if rc != FP_OK:
        raise FluidError(rc, f"cannot read level-set file {path}")
    out = np.zeros(int(dims[0]) * int(dims[1]), np.float32)
    lib().fp_read_levelset_file(str(path).encode(), ptr(dims), ptr(out))
    return out.reshape(int(dims[1]), int(dims[0]))


def default_config(**kw) -> FpConfig:
    """fp_config_default, then the given fields.  A name that is not a field of
    fp_config raises TypeError (ctypes would otherwise keep it as a plain
    attribute, and the setting would be lost without a word)."""
    cfg = FpConfig()
    lib().fp_config_default(C.byref(cfg))
    fields = {f[0] for f in FpConfig._fields_}
    for k, v in kw.items():
        if k not in fields:
            raise TypeError(f"fp_config has no field {k!r}")
        if k in ("output_template", "body_sdf"):
            setattr(cfg, k, v.encode())
        elif k == "body_pos":
            cfg.body_pos[:] = list(v)
        elif k == "solver" and isinstance(v, str):
            cfg.solver = SOLVER_NAMES[v]
        elif k == "advection" and isinstance(v, str):
            cfg.advection = {"rk3ref": ADVECT_RK3REF, "rk2": ADVECT_RK2}[v]
        elif k == "scheme" and isinstance(v, str):
            cfg.scheme = {"default": SCHEME_DEFAULT, "ref2d": SCHEME_REF2D}[v]
        elif k == "collision" and isinstance(v, str):
            cfg.collision = {"labels": COLLISION_LABELS, "sdf": COLLISION_SDF}[v]
        elif k == "body_forces" and isinstance(v, str):
            cfg.body_forces = {"face_fraction": BODY_FORCES_FACE_FRACTION, "reference": BODY_FORCES_REFERENCE}[v]
        else:
            setattr(cfg, k, v)
    return cfg


class Solver:
    """Thin owner of an ``fp_solver*`` handle with numpy in/out."""

    def __init__(self, cfg: FpConfig | None = None, **kw):
        self._h = C.c_void_p()
        self.cfg = cfg if cfg is not None else default_config(**kw)
        rc = lib().fp_create(C.byref(self.cfg), C.byref(self._h))
        if rc != FP_OK:
            raise FluidError(rc, "fp_create failed")

    def _check(self, rc):
        if rc != FP_OK:
            raise FluidError(rc, lib().fp_last_error(self._h).decode())
        return rc

    def close(self):
        if self._h:
            lib().fp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- scene
    def load_labels(self, path):
        return self._check(lib().fp_load_labels(self._h, str(path).encode()))

    def set_labels(self, labels: np.ndarray):
        lab = np.ascontiguousarray(labels, np.uint8)
        if lab.ndim == 2:
            H, W = lab.shape
            D = 1
        else:
            D, H, W = lab.shape
        return self._check(lib().fp_set_labels(self._h, ptr(lab), W, H, D))

    @property
    def dims(self):
        W, H, D = C.c_int(), C.c_int(), C.c_int()
        lib().fp_get_dims(self._h, C.byref(W), C.byref(H), C.byref(D))
        return W.value, H.value, D.value

    def load_sdf(self, path=None):
        """Body SDF from a reference SDF file, or the analytic sphere of the
        config (body_radius, body_density) when path is None."""
        return self._check(lib().fp_load_sdf(self._h, None if path is None else str(path).encode()))

    def set_labels_from_levelsets(self, solid: np.ndarray, fluid: np.ndarray):
        """Labels from solid and fluid level sets ((H, W) or (D, H, W) arrays)."""
        s = np.ascontiguousarray(solid, np.float32)
        f = np.ascontiguousarray(fluid, np.float32)
        if s.shape != f.shape or s.ndim not in (2, 3):
            raise ValueError("level sets must have the same (H, W) or (D, H, W) shape")
        D, H, W = (1,) + s.shape if s.ndim == 2 else s.shape
        return self._check(lib().fp_set_labels_from_levelsets(self._h, ptr(s), ptr(f), W, H, D))

    def scene_seabed(self, W, H, D, level=0.45, bed_base=0.15, bed_amp=0.05, seed=4, water_xmin=0.0):
        """The seabed scene labelled on the GPU (see scenes.seabed)."""
        return self._check(lib().fp_scene_seabed(self._h, W, H, D, level, bed_base, bed_amp, seed, water_xmin))

    def set_paddle(self, x_rest, amplitude, period):
        """Wave paddle: BODY where x < x_rest + amplitude sin(2 pi t / period)."""
        return self._check(lib().fp_set_paddle(self._h, x_rest, amplitude, period))

    def seed_particles(self, ppc, seed):
        return self._check(lib().fp_seed_particles(self._h, ppc, seed))

    def set_particles(self, pos, vel=None):
        pos = np.ascontiguousarray(pos, np.float32)
        v = None if vel is None else np.ascontiguousarray(vel, np.float32)
        return self._check(lib().fp_set_particles(self._h, ptr(pos), None if v is None else ptr(v), len(pos)))

    def load_ply(self, path):
        return self._check(lib().fp_load_ply(self._h, str(path).encode()))

    def save_ply(self, path, fmt=OUT_PLY):
        return self._check(lib().fp_save_ply(self._h, str(path).encode(), fmt))

    @property
    def num_particles(self):
        return lib().fp_num_particles(self._h)

    def particles(self, out=None):
        """(pos, vel) as n x 3 float32 in the order given.  out = (pos, vel)
        reuses caller arrays (pinned host memory makes the copy direct)."""
        n = self.num_particles
        if out is None:
            pos = np.empty((n, 3), np.float32)
            vel = np.empty((n, 3), np.float32)
        else:
            pos, vel = out
            for a in (pos, vel):
                if a.dtype != np.float32 or a.shape != (n, 3) or not a.flags.c_contiguous:
                    raise ValueError("out arrays must be C-contiguous float32 of shape (n, 3)")
        self._check(lib().fp_get_particles(self._h, ptr(pos), ptr(vel), n))
        return pos, vel

    # ---- stepping
    def step(self, n=1):
        return self._check(lib().fp_step(self._h, n))

    def run(self, frames):
        return self._check(lib().fp_run(self._h, frames))

    def phase(self, ph):
        return self._check(lib().fp_run_phase(self._h, ph))

    # ---- state
    def grid_shape(self, which):
        W, H, D = self.dims
        return {GRID_U: (D, H, W + 1), GRID_U_SAVED: (D, H, W + 1), GRID_V: (D, H + 1, W), GRID_V_SAVED: (D, H + 1, W),
                GRID_W: (D + 1, H, W), GRID_W_SAVED: (D + 1, H, W), GRID_P: (D, H, W), GRID_RHS: (D, H, W)}[which]

    def grid(self, which):
        shp = self.grid_shape(which)
        out = np.zeros(shp, np.float32)
        self._check(lib().fp_get_grid(self._h, which, ptr(out), out.size))
        return out

    def set_grid(self, which, data):
        a = np.ascontiguousarray(data, np.float32).reshape(-1)
        return self._check(lib().fp_set_grid(self._h, which, ptr(a), a.size))

    def grid_to_device(self, which, d_out: int, n: int):
        """Copy a grid into caller device memory at address d_out (n floats)."""
        return self._check(lib().fp_get_grid_device(self._h, which, C.c_void_p(d_out), n))

    def labels_to_device(self, d_out: int, n: int):
        return self._check(lib().fp_get_labels_device(self._h, C.c_void_p(d_out), n))

    def load_learned(self, path):
        """Weights of the learned initial guess (FP_SOLVER_PCG_LEARNED)."""
        return self._check(lib().fp_load_learned(self._h, str(path).encode()))

    def labels(self):
        W, H, D = self.dims
        out = np.zeros((D, H, W), np.uint8)
        self._check(lib().fp_get_labels(self._h, ptr(out), out.size))
        return out

    def set_body_state(self, pos=None, vel=None, omega=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (pos, vel, omega)]
        return self._check(lib().fp_set_body_state(self._h, *[None if a is None else ptr(a) for a in arrs]))

    @property
    def stream(self) -> int:
        """The solver's cudaStream_t as an integer handle."""
        return lib().fp_cuda_stream(self._h) or 0

    def set_step_log(self, path=None):
        """One JSON line of statistics per step to path (None closes the log)."""
        return self._check(lib().fp_set_step_log(self._h, None if path is None else str(path).encode()))

    def save_state(self, path):
        return self._check(lib().fp_save_state(self._h, str(path).encode()))

    def load_state(self, path):
        return self._check(lib().fp_load_state(self._h, str(path).encode()))

    def set_wait_limit(self, polls: int):
        """Polls after which a grid-barrier wait of the pressure solvers gives
        up (FP_ERR_TIMEOUT); 0 restores the default."""
        return self._check(lib().fp_set_wait_limit(self._h, int(polls)))

    def stats(self) -> dict:
        st = FpStepStats()
        lib().fp_stats(self._h, C.byref(st))
        return st.as_dict()

    def pressure_solve(self, rhs):
        W, H, D = self.dims
        b = np.ascontiguousarray(rhs, np.float32).reshape(-1)
        x = np.zeros(W * H * D, np.float32)
        it, rr = C.c_int(), C.c_double()
        rc = lib().fp_pressure_solve(self._h, ptr(b), ptr(x), b.size, C.byref(it), C.byref(rr))
        if rc not in (FP_OK, FP_ERR_SOLVER):
            self._check(rc)
        return x.reshape(D, H, W), it.value, rr.value, rc


def solve_csr_upper(offsets, cols, vals, b, tol=1e-14, max_iters=10000):
    off = np.ascontiguousarray(offsets, np.int32)
    cl = np.ascontiguousarray(cols, np.int32)
    vl = np.ascontiguousarray(vals, np.float64)
    bb = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(bb)
    it, rr = C.c_int(), C.c_double()
    rc = lib().fp_solve_csr_upper(len(bb), ptr(off), ptr(cl), ptr(vl), ptr(bb), ptr(x), tol, max_iters, C.byref(it),
                                  C.byref(rr))
    if rc != FP_OK:
        raise FluidError(rc, "fp_solve_csr_upper failed")
    return x, it.value, rr.value


FP_NOALLOC_MAX_N = 1 << 18


def solve_csr_upper_noalloc(n, d_offsets, d_cols, d_vals, d_b, d_x, tol=1e-14, max_iters=10000, stream=None):
    """fp_solve_csr_upper_noalloc on caller-owned device buffers (raw device
    addresses as ints); the solution is written to d_x.  Returns (iters,
    relres); raises FluidError on a non-zero status."""
    it, rr = C.c_int(), C.c_double()
    rc = lib().fp_solve_csr_upper_noalloc(int(n), C.c_void_p(d_offsets), C.c_void_p(d_cols), C.c_void_p(d_vals),
                                          C.c_void_p(d_b), C.c_void_p(d_x), tol, max_iters, C.byref(it),
                                          C.byref(rr), C.c_void_p(stream))
    if rc != FP_OK:
        raise FluidError(rc, "fp_solve_csr_upper_noalloc failed")
    return it.value, rr.value


def read_label_file(path, dim=3) -> np.ndarray:
    """Reference label file -> uint8 array (D, H, W) in 3D or (H, W) in 2D."""
    dims = np.zeros(3, np.int32)
    rc = lib().fp_read_label_file(str(path).encode(), dim, ptr(dims), None)
    if rc != FP_OK:
        raise FluidError(rc, f"cannot read label file {path}")
    W, H, D = map(int, dims)
    out = np.zeros(W * H * D, np.uint8)
    lib().fp_read_label_file(str(path).encode(), dim, ptr(dims), ptr(out))
    return out.reshape(D, H, W) if dim == 3 else out.reshape(H, W)


def read_ply_file(path):
    """PLY vertices -> (pos (n,3) float32, vel (n,3) float32 or None)."""
    n = C.c_int64()
    hv = C.c_int()
    rc = lib().fp_read_ply_file(str(path).encode(), C.byref(n), None, None, C.byref(hv))
    if rc != FP_OK:
        raise FluidError(rc, f"cannot read PLY {path}")
    pos = np.zeros((n.value, 3), np.float32)
    vel = np.zeros((n.value, 3), np.float32) if hv.value else None
    lib().fp_read_ply_file(str(path).encode(), C.byref(n), ptr(pos), None if vel is None else ptr(vel), C.byref(hv))
    return pos, vel


class UNet:
    """The learned preconditioner's network (fp_unet_*).  Array arguments of
    forward / loss_grad / train_step are raw DEVICE addresses (ints) of the
    real-grid arrays: labels uint8, rhs / p / x float32, W*H*D each."""

    def __init__(self, W, H, D, train=False, seed=0):
        h = C.c_void_p()
        rc = lib().fp_unet_create(W, H, D, int(bool(train)), seed, C.byref(h))
        if rc != FP_OK:
            raise FluidError(rc, "fp_unet_create failed")
        self._h = h
        self.dims = (W, H, D)

    def _check(self, rc):
        if rc != FP_OK:
            raise FluidError(rc, (lib().fp_unet_last_error(self._h) or b"").decode())
        return rc

    def close(self):
        if getattr(self, "_h", None):
            lib().fp_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def num_params() -> int:
        return int(lib().fp_unet_num_params())

    @property
    def stream(self) -> int:
        return lib().fp_unet_cuda_stream(self._h) or 0

    def params(self) -> np.ndarray:
        out = np.zeros(self.num_params(), np.float32)
        self._check(lib().fp_unet_get_params(self._h, ptr(out), out.size))
        return out

    def set_params(self, w):
        a = np.ascontiguousarray(w, np.float32)
        return self._check(lib().fp_unet_set_params(self._h, ptr(a), a.size))

    def save(self, path):
        return self._check(lib().fp_unet_save(self._h, str(path).encode()))

    def load(self, path):
        return self._check(lib().fp_unet_load(self._h, str(path).encode()))

    def forward(self, d_labels: int, d_rhs: int, d_x: int):
        return self._check(lib().fp_unet_forward(self._h, C.c_void_p(d_labels), C.c_void_p(d_rhs), C.c_void_p(d_x)))

    def loss_grad(self, d_labels: int, d_rhs: int, d_p: int):
        loss = C.c_double()
        g = np.zeros(self.num_params(), np.float32)
        self._check(lib().fp_unet_loss_grad(self._h, C.c_void_p(d_labels), C.c_void_p(d_rhs), C.c_void_p(d_p),
                                            C.byref(loss), ptr(g)))
        return loss.value, g

    def train_step(self, d_labels: int, d_rhs: int, d_p: int, lr: float, want_loss=False):
        loss = C.c_double()
        self._check(lib().fp_unet_train_step(self._h, C.c_void_p(d_labels), C.c_void_p(d_rhs), C.c_void_p(d_p),
                                             lr, C.byref(loss) if want_loss else None))
        return loss.value if want_loss else None
