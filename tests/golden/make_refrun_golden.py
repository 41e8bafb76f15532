"""Make tests/golden/refrun_3d.npz: phases of the reference's own 3D solver,
run on a GPU on a seeded scene.

TEST INFRASTRUCTURE ONLY.  Needs oracle/_ref/libref3d.so, built here by
``FLUIDPRJCT_REFERENCE=<checkout> make -C oracle/refrun`` from the reference's
unmodified src/FluidSim/FluidSolver3D.cu and utility.cu (with a compile-only
cuDSS stand-in), and a CUDA GPU to run it on.  Run from the repository root:

    python tests/golden/make_refrun_golden.py [out.npz]

The scene: a 20 x 16 x 12 grid, dx = 0.05, one-cell SOLID walls, an interior
SOLID block, a FLUID box x < 0.62, y < 0.55, z < 0.5 seeded with 8 particles
per cell (oracle.seed3d, seed 11) with velocities uniform in [-0.6, 0.6]
(seed 11).  The reference runs labelGrid, particlesToGrid, saveVelocities
and applyForces (dt = 0.004), then gridToParticles(0.05) and
advectParticles(0.1) with every face grid (u, v, w, u*, v*, w*) replaced by
values uniform in [-1, 1] (numpy default_rng(5), in that order).  Its labels,
its grids after P2G and after the forces, and its particles after G2P and
advection are stored with the inputs.
"""
import ctypes as C
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

W, H, D, DX, DT, ALPHA, CFL = 20, 16, 12, 0.05, 0.004, 0.05, 0.1


def scene():
    from fluidprjct_b200 import scenes
    from oracle import oracle as O
    lab = scenes.box_3d(W, H, D, DX, 0.62, 0.55, 0.5)
    lab[2:5, 2:4, 9:12] = 0  # an interior SOLID block
    pos = O.seed3d(lab, DX, 8, 11)
    vel = np.random.default_rng(11).uniform(-0.6, 0.6, pos.shape).astype(np.float32)
    rng = np.random.default_rng(5)
    nu, nv, nw = (W + 1) * H * D, W * (H + 1) * D, W * H * (D + 1)
    grids = [rng.uniform(-1, 1, n).astype(np.float32) for n in (nu, nv, nw, nu, nv, nw)]
    return lab, pos, vel, grids


def main(out):
    from fluidprjct_b200 import scenes
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref3d.so"))
    P = C.c_void_p
    lib.ref3d_run.argtypes = [C.c_char_p, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int64, P, P, P, P, P, P,
                              P, P]
    lab, pos, vel, grids = scene()
    n = len(pos)
    nu, nv, nw = (W + 1) * H * D, W * (H + 1) * D, W * H * (D + 1)
    g_in = np.ascontiguousarray(np.concatenate(grids))
    labels = np.zeros(W * H * D, np.int32)
    p2g = np.zeros(nu + nv + nw, np.float32)
    forces = np.zeros(nu + nv + nw, np.float32)
    pos_out = np.zeros_like(pos)
    vel_out = np.zeros_like(vel)
    p = lambda a: a.ctypes.data_as(P)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "InputData"))  # init() writes InputData/particles_-1.ply
        path = os.path.join(tmp, "labels.txt")
        scenes.write_labels3d(path, lab)
        os.chdir(tmp)
        try:
            rc = lib.ref3d_run(path.encode(), DX, DT, ALPHA, CFL, n, p(pos), p(vel), p(g_in), p(labels), p(p2g),
                               p(forces), p(pos_out), p(vel_out))
        finally:
            os.chdir(cwd)
    if rc != 0:
        sys.exit(f"ref3d_run failed: {rc}")
    np.savez_compressed(out, dims=np.array([W, H, D]), dx=DX, dt=DT, alpha=ALPHA, cfl=CFL,
                        labels_in=lab, pos_in=pos, vel_in=vel, g2p_in=g_in,
                        labels=labels.reshape(D, H, W).astype(np.uint8),
                        p2g=p2g, forces=forces, pos_out=pos_out, vel_out=vel_out)
    print(f"{out}: {n} particles, {int((labels == 1).sum())} FLUID cells")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "refrun_3d.npz"))
