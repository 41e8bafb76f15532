"""The reference's own 2D step (scheme ref2d, FluidSolver2D.cu) on the GPU
against the oracle's restatement (oracle/ref2d_oracle.cpp).

Every phase but the pressure solve is bit-exact: the kernels use the same
FP32 operation order without FMA contraction, and P2G sums each face's
contributions in particle order.  The pressure solve (MG-PCG to 1e-9 here,
FP64 CG in the oracle) agrees within 1e-5 relative L2, and the oracle then
continues from the GPU's pressure so the later phases stay comparable bit
for bit.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _scene(O, n=32, ppc=4, seed=0, dt=0.005, jitter=0.3, alpha=0.05, extrapolate=0):
    from fluidprjct_b200 import capi, scenes
    lab = scenes.dam_break_2d(n)
    dx = 1.0 / n
    pos = O.seed2d(lab, dx, ppc, seed)
    vel = np.zeros_like(pos)
    vel[:, :2] = np.random.default_rng(seed).uniform(-jitter, jitter, (len(pos), 2))
    s = capi.Solver(dim=2, dx=dx, dt=dt, pic_weight=alpha, solver="pcg_mg", tol=1e-9, scheme="ref2d",
                    output_format=capi.OUT_NONE, extrapolate=extrapolate)
    s.set_labels(lab)
    s.set_particles(pos, vel)
    o = O.Ref2D(n, n, dx, dt, pic_weight=alpha, tol=1e-13)
    o.set_extrapolate(extrapolate)
    o.set_labels(lab)
    o.set_particles(pos, vel)
    return s, o, lab


def _same(a, b):
    a = np.asarray(a, np.float32).ravel()
    b = np.asarray(b, np.float32).ravel()
    return a.shape == b.shape and np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("extrapolate", [0, 1])
def test_ref2d_phases_bit_exact(O, extrapolate):
    """With extrapolate = 1 the step's two commented-out extrapolateGridFluidData
    calls run too (after P2G, and between G2P and advection)."""
    from fluidprjct_b200 import capi
    s, o, lab = _scene(O, extrapolate=extrapolate)
    for k in range(3):  # three steps, phase by phase
        s.phase(capi.PHASE_LABEL); o.phase(O.PH_LABEL)
        assert np.array_equal(s.labels().reshape(o.labels().shape), o.labels())
        s.phase(capi.PHASE_P2G); o.phase(O.PH_P2G)
        for g in (capi.GRID_U, capi.GRID_V):
            assert _same(s.grid(g), o.grid(g)), (k, g)
        s.phase(capi.PHASE_SAVE); o.phase(O.PH_SAVE)
        s.phase(capi.PHASE_FORCES); o.phase(O.PH_FORCES)
        for g in (capi.GRID_U, capi.GRID_V, capi.GRID_U_SAVED, capi.GRID_V_SAVED):
            assert _same(s.grid(g), o.grid(g)), (k, g)
        s.phase(capi.PHASE_PRESSURE); o.phase(O.PH_PRESSURE)
        p = s.grid(capi.GRID_P)
        assert rel_l2(p, o.grid(O.GRID_P)) <= 1e-5
        o.set_grid(O.GRID_P, p.astype(np.float64))
        s.phase(capi.PHASE_PROJECT); o.phase(O.PH_PROJECT)
        for g in (capi.GRID_U, capi.GRID_V):
            assert _same(s.grid(g), o.grid(g)), (k, g)
        assert np.any(s.grid(capi.GRID_U) == O.VEL_UNKNOWN)
        for ph_s, ph_o in ((capi.PHASE_G2P, O.PH_G2P), (capi.PHASE_ADVECT, O.PH_ADVECT),
                           (capi.PHASE_CLEANUP, O.PH_CLEANUP)):
            s.phase(ph_s); o.phase(ph_o)
            pg, vg = s.particles()
            po, vo = o.particles()
            assert len(pg) == len(po)
            assert _same(pg[:, :2], po[:, :2]) and _same(vg[:, :2], vo[:, :2]), (k, ph_s)
    assert s.stats()["advect_capped"] == 0


def test_ref2d_cleanup_deletes_like_the_oracle(O):
    """Particles outside the grid, or in a SOLID cell with no SOLID or AIR
    neighbour, are erased with the order kept (cleanUpParticles, :1171-1204)."""
    from fluidprjct_b200 import capi
    s, o, lab = _scene(O, n=16, ppc=2)
    pos, vel = s.particles()
    rng = np.random.default_rng(1)
    pick = rng.choice(len(pos), 40, replace=False)
    pos[pick[:10], 0] = 1.3          # right of the grid
    pos[pick[10:20], 1] = -0.2       # below it: y in (-dx, 0) stays in row 0, further is deleted
    pos[pick[20:30], 0] = -0.01      # x in (-dx, 0): column 0 (SOLID), projected
    s.set_particles(pos, vel)
    o.set_particles(pos, vel)
    s.phase(capi.PHASE_CLEANUP); o.phase(O.PH_CLEANUP)
    pg, vg = s.particles()
    po, vo = o.particles()
    assert len(pg) == len(po) < len(pos)
    assert s.stats()["particles_removed"] == len(pos) - len(pg) == o.stats()["removed"]
    assert _same(pg[:, :2], po[:, :2]) and _same(vg[:, :2], vo[:, :2])


def test_ref2d_steps_track_the_oracle(O):
    """Whole steps (fused kernels) against the oracle's step.  The pressure
    solves differ at the 1e-9 level, so the states are compared with a
    tolerance after 20 steps of the config-1 dam break at 32^2."""
    s, o, lab = _scene(O, jitter=0.0)
    n0 = s.num_particles
    s.step(20)
    o.step(20)
    st = s.stats()
    pg, vg = s.particles()
    po, vo = o.particles()
    assert st["solve_status"] == 0 and st["advect_capped"] == 0
    assert len(pg) == len(po) == n0
    assert np.abs(pg - po).max() <= 1e-4
    assert rel_l2(vg, vo) <= 1e-4
    assert st["kernel_launches"] > 0


def test_ref2d_dam_break_config(tmp_path):
    """Config 1 (64^2, dx = 1/64, 4 ppc seed 0, dt = 0.005, FLIP 0.95) for
    100 steps under the reference's 2D step, with fp_run's per-step frames
    (FluidSolver2D::run, :1333-1342)."""
    from fluidprjct_b200 import capi, scenes
    lab = scenes.dam_break_2d(64)
    s = capi.Solver(dim=2, dx=1 / 64, dt=0.005, pic_weight=0.05, solver="pcg_mg", tol=1e-6, scheme="ref2d",
                    output_format=capi.OUT_PLY, output_template=str(tmp_path / "particles_"))
    s.set_labels(lab)
    s.seed_particles(4, 0)
    p0, _ = s.particles()
    assert len(p0) == 3100
    s.run(100)
    st = s.stats()
    p, v = s.particles()
    assert st["step"] == 100 and st["solve_status"] == 0 and st["residual"] <= 1e-6
    assert sorted(f.name for f in tmp_path.iterdir()) == sorted(f"particles_{i}.ply" for i in range(100))
    assert np.isfinite(p).all() and len(p) <= 3100
    assert p[:, 1].mean() < p0[:, 1].mean()


def test_ref2d_without_particles_and_config_checks():
    from fluidprjct_b200 import capi, scenes
    lab = scenes.dam_break_2d(16)
    s = capi.Solver(dim=2, dx=1 / 16, dt=0.005, scheme="ref2d", output_format=capi.OUT_NONE)
    s.set_labels(lab)
    s.set_particles(np.zeros((0, 3), np.float32))
    s.step(2)  # no FLUID cell: the solve reports it, the step goes on
    assert s.num_particles == 0 and s.stats()["solve_status"] == capi.FP_ERR_NO_FLUID
