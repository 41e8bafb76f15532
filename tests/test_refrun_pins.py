"""The oracle and the GPU path pinned by outputs of the reference's own code.

tests/golden/refrun_3d.npz holds phases of the unmodified reference 3D solver
(src/FluidSim/FluidSolver3D.cu, compiled for sm_100a with a compile-only cuDSS
stand-in and run on a B200 by tests/golden/make_refrun_golden.py): its labels
(labelGrid, :340-397), its face grids after particlesToGrid (:438-685) and
after applyForces (:700-761), and its particles after gridToParticles
(:803-1039) and advectParticles (:1241-1357, RK3) from given grids.

The reference sums P2G with float atomics in an unspecified order, so its
grids are reproducible only to rounding: the bars are 1e-6 relative L2 for
grids and velocities (FP32 rounding is ~6e-8), labels bit-exact, and 99.9 %
of positions within 1e-5 dx (a substep boundary can flip on a rounding).
The CPU test checks the oracle (FP32 mode, the reference's expression
order); the GPU test checks the product through its C ABI.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

FIX = os.path.join(GOLDEN, "refrun_3d.npz")


def _fixture():
    z = np.load(FIX)
    W, H, D = (int(x) for x in z["dims"])
    nu, nv, nw = (W + 1) * H * D, W * (H + 1) * D, W * H * (D + 1)
    split = lambda a: (a[:nu], a[nu:nu + nv], a[nu + nv:nu + nv + nw])
    g = z["g2p_in"]
    g2p = split(g[:nu + nv + nw]) + split(g[nu + nv + nw:])
    return z, (W, H, D), split(z["p2g"]), split(z["forces"]), g2p


def _check(labels, p2g, forces, vel, pos, z, dx):
    assert np.array_equal(labels, z["labels"])
    _, _, ref_p2g, ref_forces, _ = _fixture()
    for a, b in zip(p2g, ref_p2g):
        assert rel_l2(a, b) <= 1e-6, rel_l2(a, b)
    for a, b in zip(forces, ref_forces):
        assert rel_l2(a, b) <= 1e-6, rel_l2(a, b)
    assert rel_l2(vel, z["vel_out"]) <= 1e-6, rel_l2(vel, z["vel_out"])
    err = np.abs(np.asarray(pos, np.float64) - z["pos_out"]).max(axis=1)
    assert np.mean(err <= 1e-5 * dx) >= 0.999, np.sort(err)[-10:]
    assert err.max() <= 0.6 * dx


def test_fixture_is_a_nontrivial_reference_run():
    z, (W, H, D), p2g, forces, _ = _fixture()
    assert z["labels"].shape == (D, H, W) and int((z["labels"] == 1).sum()) > 300
    assert len(z["pos_in"]) > 2000
    assert np.abs(p2g[0]).max() > 0.1 and np.abs(p2g[1]).max() > 0.1
    moved = np.abs(z["pos_out"] - z["pos_in"]).max(axis=1)
    assert moved.max() > 0.05 * float(z["dx"])
    # forces added dt * g to every v face (the reference's x > INT_MIN test)
    assert np.allclose(forces[1] - p2g[1], np.float32(z["dt"]) * np.float32(-9.81), atol=1e-6)


def test_oracle_matches_the_reference_run(O):
    z, (W, H, D), _, _, g2p = _fixture()
    dx = float(z["dx"])
    o = O.Sim3(W, H, D, dx, float(z["dt"]), fp64=False, pic_weight=float(z["alpha"]), cfl=float(z["cfl"]))
    o.set_labels(z["labels_in"])
    o.set_particles(z["pos_in"], z["vel_in"])
    o.phase(O.PH_LABEL)
    labels = o.labels()
    o.phase(O.PH_P2G)
    p2g = [o.grid(g) for g in (O.GRID_U, O.GRID_V, O.GRID_W)]
    o.phase(O.PH_SAVE)
    o.phase(O.PH_FORCES)
    forces = [o.grid(g) for g in (O.GRID_U, O.GRID_V, O.GRID_W)]
    for g, a in zip((O.GRID_U, O.GRID_V, O.GRID_W, O.GRID_US, O.GRID_VS, O.GRID_WS), g2p):
        o.set_grid(g, a.astype(np.float64))
    o.phase(O.PH_G2P)
    o.phase(O.PH_ADVECT)
    pos, vel = o.particles()
    _check(labels, p2g, forces, vel, pos, z, dx)


@pytest.mark.gpu
def test_gpu_matches_the_reference_run():
    from fluidprjct_b200 import capi
    z, (W, H, D), _, _, g2p = _fixture()
    dx = float(z["dx"])
    s = capi.Solver(dx=dx, dt=float(z["dt"]), pic_weight=float(z["alpha"]), cfl=float(z["cfl"]),
                    advection="rk3ref")
    s.set_labels(z["labels_in"])
    s.set_particles(z["pos_in"], z["vel_in"])
    s.phase(capi.PHASE_LABEL)
    labels = s.labels()
    s.phase(capi.PHASE_P2G)
    p2g = [s.grid(g).ravel() for g in (capi.GRID_U, capi.GRID_V, capi.GRID_W)]
    s.phase(capi.PHASE_SAVE)
    s.phase(capi.PHASE_FORCES)
    forces = [s.grid(g).ravel() for g in (capi.GRID_U, capi.GRID_V, capi.GRID_W)]
    for g, a in zip((capi.GRID_U, capi.GRID_V, capi.GRID_W, capi.GRID_U_SAVED, capi.GRID_V_SAVED,
                     capi.GRID_W_SAVED), g2p):
        s.set_grid(g, a)
    s.phase(capi.PHASE_G2P)
    s.phase(capi.PHASE_ADVECT)
    pos, vel = s.particles()
    _check(labels, p2g, forces, vel, pos, z, dx)
    s.close()
