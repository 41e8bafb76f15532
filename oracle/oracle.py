"""ctypes binding of the CPU oracle (``oracle/fluid_oracle.cpp``,
``oracle/ref2d_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline / reference legs, never by the product package.
The oracle restates Ship-Vano/FluidPrjct's 3D PIC/FLIP step
(``src/FluidSim/FluidSolver3D.cu``, class ``Sim3``) and its own 2D step
(``src/FluidSim/FluidSolver2D.cu``, class ``Ref2D``) on the CPU; the headers
of the two C++ files give the arithmetic modes and the pins.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

GRID_U, GRID_V, GRID_W, GRID_US, GRID_VS, GRID_WS, GRID_P = range(7)
PH_LABEL, PH_P2G, PH_SAVE, PH_FORCES, PH_PRESSURE, PH_PROJECT, PH_BODY, PH_G2P, PH_ADVECT, PH_CLEANUP = range(10)
VEL_UNKNOWN = float(np.float32(-2.0 ** 31))  # INT_MIN stored in a float grid (utility.cuh:56)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, OpenMP) and return the .so path."""
    srcs = [os.path.join(_HERE, f) for f in ("fluid_oracle.cpp", "ref2d_oracle.cpp")]
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < max(map(os.path.getmtime, srcs)):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        P, I, D, I64, U32 = C.c_void_p, C.c_int, C.c_double, C.c_int64, C.c_uint32
        L.or_read_labels3d.argtypes = [C.c_char_p, P, P]
        L.or_read_labels2d.argtypes = [C.c_char_p, P, P]
        L.or_seed3d.argtypes = [P, I, I, I, C.c_float, I, U32, P]
        L.or_seed3d.restype = I64
        L.or_bin3d.argtypes = [P, I64, I, I, I, C.c_float, P, P]
        L.or_seed2d.argtypes = [P, I, I, C.c_float, I, U32, P]
        L.or_seed2d.restype = I64
        L.or_build_csr_upper.argtypes = [P, I, I, I, P, P, P, P, P]
        L.or_cg_csr_upper.argtypes = [I, P, P, P, P, P, D, I, P]
        L.or3_create.argtypes = [I, I, I, D, D, I]
        L.or3_create.restype = P
        L.or3_destroy.argtypes = [P]
        L.or3_set_params.argtypes = [P, D, D, D, I]
        L.or3_set_body.argtypes = [P, P, P, P]
        L.or3_set_rk2.argtypes = [P, I]
        L.or3_set_collision.argtypes = [P, I]
        L.or3_set_sphere.argtypes = [P, P, D, D]
        L.or3_set_paddle.argtypes = [P, D, D, D]
        L.or3_set_extrap.argtypes = [P, I]
        L.or3_set_ref_forces.argtypes = [P, I]
        L.or3_ref_forces.argtypes = [P, P]
        L.or2r_set_extrap.argtypes = [P, I]
        L.or3_body_state.argtypes = [P, P]
        L.or3_body_force.argtypes = [P, P]
        L.or3_set_labels.argtypes = [P, P]
        L.or3_get_labels.argtypes = [P, P]
        L.or3_set_particles.argtypes = [P, I64, P, P]
        L.or3_num_particles.argtypes = [P]
        L.or3_num_particles.restype = I64
        L.or3_get_particles.argtypes = [P, P, P]
        L.or3_grid_len.argtypes = [P, I]
        L.or3_grid_len.restype = I64
        L.or3_grid_io.argtypes = [P, I, P, I]
        L.or3_phase.argtypes = [P, I]
        L.or3_step.argtypes = [P, I]
        L.or3_rhs.argtypes = [P, P]
        L.or3_solve.argtypes = [P, P, P]
        L.or3_apply.argtypes = [P, P, P]
        L.or3_stats.argtypes = [P, P]
        L.or_num_threads.restype = I
        L.or2r_create.argtypes = [I, I, D, D, I]
        L.or2r_create.restype = P
        L.or2r_destroy.argtypes = [P]
        L.or2r_set_params.argtypes = [P, D, D, I]
        L.or2r_set_labels.argtypes = [P, P]
        L.or2r_get_labels.argtypes = [P, P]
        L.or2r_set_particles.argtypes = [P, I64, P, P]
        L.or2r_num_particles.argtypes = [P]
        L.or2r_num_particles.restype = I64
        L.or2r_get_particles.argtypes = [P, P, P]
        L.or2r_grid_len.argtypes = [P, I]
        L.or2r_grid_len.restype = I64
        L.or2r_grid_io.argtypes = [P, I, P, I]
        L.or2r_phase.argtypes = [P, I]
        L.or2r_step.argtypes = [P, I]
        L.or2r_stats.argtypes = [P, P]
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def read_labels3d(path: str) -> np.ndarray:
    """Labels as uint8 array of shape (D, H, W) (index i + j*W + k*W*H)."""
    dims = np.zeros(3, np.int32)
    rc = lib().or_read_labels3d(path.encode(), _p(dims), None)
    if rc:
        raise ValueError(f"bad label file {path}: {rc}")
    W, H, D = map(int, dims)
    out = np.zeros(W * H * D, np.uint8)
    rc = lib().or_read_labels3d(path.encode(), _p(dims), _p(out))
    if rc:
        raise ValueError(f"bad label file {path}: {rc}")
    return out.reshape(D, H, W)


def read_labels2d(path: str) -> np.ndarray:
    dims = np.zeros(2, np.int32)
    rc = lib().or_read_labels2d(path.encode(), _p(dims), None)
    if rc:
        raise ValueError(f"bad label file {path}: {rc}")
    W, H = map(int, dims)
    out = np.zeros(W * H, np.uint8)
    rc = lib().or_read_labels2d(path.encode(), _p(dims), _p(out))
    if rc:
        raise ValueError(f"bad label file {path}: {rc}")
    return out.reshape(H, W)


def seed3d(labels: np.ndarray, dx: float, ppc: int, seed: int) -> np.ndarray:
    lab = np.ascontiguousarray(labels, np.uint8)
    D, H, W = lab.shape
    n = lib().or_seed3d(_p(lab), W, H, D, dx, ppc, seed, None)
    pos = np.zeros((n, 3), np.float32)
    lib().or_seed3d(_p(lab), W, H, D, dx, ppc, seed, _p(pos))
    return pos


def seed2d(labels: np.ndarray, dx: float, ppc: int, seed: int) -> np.ndarray:
    lab = np.ascontiguousarray(labels, np.uint8)
    H, W = lab.shape
    n = lib().or_seed2d(_p(lab), W, H, dx, ppc, seed, None)
    pos = np.zeros((n, 3), np.float32)
    lib().or_seed2d(_p(lab), W, H, dx, ppc, seed, _p(pos))
    return pos


def bin3d(pos: np.ndarray, dims, dx: float):
    """Cell key per particle and per-cell counts (floorf(p/dx), clamped)."""
    W, H, D = dims
    pos = np.ascontiguousarray(pos, np.float32)
    keys = np.zeros(len(pos), np.int32)
    counts = np.zeros(W * H * D, np.int32)
    lib().or_bin3d(_p(pos), len(pos), W, H, D, dx, _p(keys), _p(counts))
    return keys, counts


def build_csr_upper(labels: np.ndarray):
    lab = np.ascontiguousarray(labels, np.uint8)
    D, H, W = lab.shape
    n, nnz = C.c_int(), C.c_int()
    lib().or_build_csr_upper(_p(lab), W, H, D, C.byref(n), C.byref(nnz), None, None, None)
    off = np.zeros(n.value + 1, np.int32)
    cols = np.zeros(nnz.value, np.int32)
    vals = np.zeros(nnz.value, np.float32)
    lib().or_build_csr_upper(_p(lab), W, H, D, C.byref(n), C.byref(nnz), _p(off), _p(cols), _p(vals))
    return off, cols, vals


def cg_csr_upper(off, cols, vals, b, tol=1e-14, maxit=10000):
    off = np.ascontiguousarray(off, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    vals = np.ascontiguousarray(vals, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b)
    rr = C.c_double()
    it = lib().or_cg_csr_upper(len(b), _p(off), _p(cols), _p(vals), _p(b), _p(x), tol, maxit, C.byref(rr))
    return x, it, rr.value


class Sim3:
    """Oracle 3D simulation (fp64=False: reference FP32 order; True: FP64)."""

    def __init__(self, W, H, D, dx, dt, fp64=False, pic_weight=0.05, cfl=0.1, tol=1e-12, maxit=100000, rk2=False):
        self.W, self.H, self.D = W, H, D
        self.h = lib().or3_create(W, H, D, dx, dt, int(fp64))
        lib().or3_set_params(self.h, pic_weight, cfl, tol, maxit)
        lib().or3_set_rk2(self.h, int(rk2))

    def close(self):
        if self.h:
            lib().or3_destroy(self.h)
            self.h = None

    __del__ = close

    def set_params(self, pic_weight, cfl=0.1, tol=1e-12, maxit=100000):
        lib().or3_set_params(self.h, pic_weight, cfl, tol, maxit)

    def set_body(self, vel, omega, com):
        a = [np.ascontiguousarray(x, np.float64) for x in (vel, omega, com)]
        lib().or3_set_body(self.h, *[_p(x) for x in a])

    def set_sphere(self, pos, radius, mass):
        a = np.ascontiguousarray(pos, np.float64)
        lib().or3_set_sphere(self.h, _p(a), radius, mass)

    def set_paddle(self, x_rest, amplitude, period):
        lib().or3_set_paddle(self.h, x_rest, amplitude, period)

    def set_collision(self, sdf):
        """SDF collision projection against the body (True) or the
        reference's label search alone (False)."""
        lib().or3_set_collision(self.h, int(bool(sdf)))

    def set_extrapolate(self, layers):
        """Velocity extrapolation layers between G2P and advection (0 = off)."""
        lib().or3_set_extrap(self.h, layers)

    def set_reference_forces(self, on=True):
        """The reference's panel drag/lift and voxel buoyancy in the body phase."""
        lib().or3_set_ref_forces(self.h, int(bool(on)))

    def reference_forces(self):
        """Force, torque, body volume, submerged volume of the last body phase."""
        out = np.zeros(8, np.float64)
        lib().or3_ref_forces(self.h, _p(out))
        return out

    def body_state(self):
        out = np.zeros(18, np.float64)
        lib().or3_body_state(self.h, _p(out))
        return {"pos": out[0:3], "vel": out[3:6], "omega": out[6:9], "angles": out[9:12], "force": out[12:15],
                "torque": out[15:18]}

    def body_force(self):
        out = np.zeros(6, np.float64)
        lib().or3_body_force(self.h, _p(out))
        return out

    def set_labels(self, labels):
        lab = np.ascontiguousarray(labels, np.uint8).reshape(-1)
        assert lab.size == self.W * self.H * self.D
        lib().or3_set_labels(self.h, _p(lab))

    def labels(self):
        out = np.zeros(self.W * self.H * self.D, np.uint8)
        lib().or3_get_labels(self.h, _p(out))
        return out.reshape(self.D, self.H, self.W)

    def set_particles(self, pos, vel=None):
        pos = np.ascontiguousarray(pos, np.float32)
        v = None if vel is None else np.ascontiguousarray(vel, np.float32)
        lib().or3_set_particles(self.h, len(pos), _p(pos), None if v is None else _p(v))

    def particles(self):
        n = lib().or3_num_particles(self.h)
        pos = np.zeros((n, 3), np.float64)
        vel = np.zeros((n, 3), np.float64)
        lib().or3_get_particles(self.h, _p(pos), _p(vel))
        return pos, vel

    def grid(self, which):
        n = lib().or3_grid_len(self.h, which)
        out = np.zeros(n, np.float64)
        lib().or3_grid_io(self.h, which, _p(out), 0)
        return out

    def set_grid(self, which, data):
        n = lib().or3_grid_len(self.h, which)
        a = np.ascontiguousarray(data, np.float64).reshape(-1)
        assert a.size == n
        lib().or3_grid_io(self.h, which, _p(a), 1)

    def phase(self, ph):
        return lib().or3_phase(self.h, ph)

    def step(self, n=1):
        return lib().or3_step(self.h, n)

    def rhs(self):
        out = np.zeros(self.W * self.H * self.D, np.float64)
        lib().or3_rhs(self.h, _p(out))
        return out

    def solve(self, b):
        b = np.ascontiguousarray(b, np.float64).reshape(-1)
        x = np.zeros_like(b)
        it = lib().or3_solve(self.h, _p(b), _p(x))
        return x, it

    def apply(self, x):
        x = np.ascontiguousarray(x, np.float64).reshape(-1)
        out = np.zeros_like(x)
        lib().or3_apply(self.h, _p(x), _p(out))
        return out

    def stats(self):
        out = np.zeros(3, np.float64)
        lib().or3_stats(self.h, _p(out))
        return {"iters": int(out[0]), "relres": float(out[1]), "nf": int(out[2])}


class Ref2D:
    """Oracle of the reference's own 2D step (FluidSolver2D.cu); fp64=False
    follows its FP32 expression order.  Phases as in ``Sim3`` plus
    PH_CLEANUP; labels are (H, W), particles n x 3 with z ignored."""

    def __init__(self, W, H, dx, dt, fp64=False, pic_weight=0.5, tol=1e-12, maxit=100000):
        self.W, self.H = W, H
        self.h = lib().or2r_create(W, H, dx, dt, int(fp64))
        lib().or2r_set_params(self.h, pic_weight, tol, maxit)

    def close(self):
        if self.h:
            lib().or2r_destroy(self.h)
            self.h = None

    __del__ = close

    def set_labels(self, labels):
        lab = np.ascontiguousarray(labels, np.uint8).reshape(-1)
        assert lab.size == self.W * self.H
        lib().or2r_set_labels(self.h, _p(lab))

    def set_extrapolate(self, on):
        """The step's commented-out extrapolateGridFluidData calls."""
        lib().or2r_set_extrap(self.h, int(bool(on)))

    def labels(self):
        out = np.zeros(self.W * self.H, np.uint8)
        lib().or2r_get_labels(self.h, _p(out))
        return out.reshape(self.H, self.W)

    def set_particles(self, pos, vel=None):
        pos = np.ascontiguousarray(pos, np.float32)
        v = None if vel is None else np.ascontiguousarray(vel, np.float32)
        lib().or2r_set_particles(self.h, len(pos), _p(pos), None if v is None else _p(v))

    def particles(self):
        n = lib().or2r_num_particles(self.h)
        pos = np.zeros((n, 3), np.float64)
        vel = np.zeros((n, 3), np.float64)
        lib().or2r_get_particles(self.h, _p(pos), _p(vel))
        return pos, vel

    def grid(self, which):
        n = lib().or2r_grid_len(self.h, which)
        out = np.zeros(n, np.float64)
        lib().or2r_grid_io(self.h, which, _p(out), 0)
        return out

    def set_grid(self, which, data):
        n = lib().or2r_grid_len(self.h, which)
        a = np.ascontiguousarray(data, np.float64).reshape(-1)
        assert a.size == n
        lib().or2r_grid_io(self.h, which, _p(a), 1)

    def phase(self, ph):
        return lib().or2r_phase(self.h, ph)

    def step(self, n=1):
        return lib().or2r_step(self.h, n)

    def stats(self):
        out = np.zeros(4, np.int64)
        lib().or2r_stats(self.h, _p(out))
        return {"nf": int(out[0]), "cg_iters": int(out[1]), "removed": int(out[2]), "capped": int(out[3])}


def num_threads() -> int:
    return lib().or_num_threads()
