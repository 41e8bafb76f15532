"""2D path (grids with depth 1) on the GPU against the oracle."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _pair2d(O, n=32, ppc=4, seed=0, dt=0.005, solver="pcg_mixed", tol=1e-9):
    from fluidprjct_b200 import capi, scenes
    lab = scenes.dam_break_2d(n)
    dx = 1.0 / n
    pos = O.seed2d(lab, dx, ppc, seed)
    vel = np.zeros_like(pos)
    vel[:, :2] = np.random.default_rng(seed).uniform(-0.3, 0.3, (len(pos), 2))
    s = capi.Solver(dim=2, dx=dx, dt=dt, pic_weight=0.05, solver=solver, tol=tol)
    s.set_labels(lab)
    s.set_particles(pos, vel)
    o = O.Sim3(n, n, 1, dx, dt, fp64=False, pic_weight=0.05, tol=1e-13)
    o.set_labels(lab[None])
    o.set_particles(pos, vel)
    return s, o, lab, pos


def test_2d_seeding_matches_oracle(O):
    from fluidprjct_b200 import capi, scenes
    lab = scenes.dam_break_2d(64)
    s = capi.Solver(dim=2, dx=1 / 64, dt=0.005)
    s.set_labels(lab)
    s.seed_particles(4, 0)
    pos, _ = s.particles()
    assert np.array_equal(pos, O.seed2d(lab, 1 / 64, 4, 0))
    assert len(pos) == 3100


def test_2d_phases_match_oracle(O):
    from fluidprjct_b200 import capi
    s, o, lab, pos = _pair2d(O)
    for ph_s, ph_o in ((capi.PHASE_LABEL, O.PH_LABEL), (capi.PHASE_P2G, O.PH_P2G), (capi.PHASE_SAVE, O.PH_SAVE),
                       (capi.PHASE_FORCES, O.PH_FORCES)):
        s.phase(ph_s)
        o.phase(ph_o)
    assert np.array_equal(s.labels(), o.labels())
    for g in (capi.GRID_U, capi.GRID_V):
        assert rel_l2(s.grid(g), o.grid(g)) <= 1e-5
    s.phase(capi.PHASE_PRESSURE)
    o.phase(O.PH_PRESSURE)
    assert rel_l2(s.grid(capi.GRID_P), o.grid(O.GRID_P)) <= 1e-5
    o.set_grid(O.GRID_P, s.grid(capi.GRID_P).astype(np.float64))
    s.phase(capi.PHASE_PROJECT)
    o.phase(O.PH_PROJECT)
    for g in (capi.GRID_U, capi.GRID_V, capi.GRID_W):
        assert rel_l2(s.grid(g), o.grid(g)) <= 1e-5
    assert not s.grid(capi.GRID_W).any()
    s.phase(capi.PHASE_G2P); o.phase(O.PH_G2P)
    s.phase(capi.PHASE_ADVECT); o.phase(O.PH_ADVECT)
    pg, vg = s.particles()
    po, vo = o.particles()
    assert rel_l2(vg, vo) <= 1e-5
    assert np.mean(np.abs(pg - po).max(axis=1) <= 1e-5 / 32) >= 0.999
    assert np.all(pg[:, 2] == 0)


@pytest.mark.parametrize("solver", ["pcg_mixed", "pcg_mg"])
def test_2d_dam_break_config(O, solver):
    """The plain 2D dam break: 64^2, dx = 1/64, 4 ppc (seed 0), dt = 0.005,
    FLIP 0.95, 100 steps, PCG to 1e-6."""
    from fluidprjct_b200 import capi, scenes
    lab = scenes.dam_break_2d(64)
    s = capi.Solver(dim=2, dx=1 / 64, dt=0.005, pic_weight=0.05, solver=solver, tol=1e-6)
    s.set_labels(lab)
    s.seed_particles(4, 0)
    p0, _ = s.particles()
    s.step(100)
    st = s.stats()
    p, v = s.particles()
    assert st["solve_status"] == 0 and st["residual"] <= 1e-6
    assert len(p) == 3100 and np.isfinite(p).all() and np.all(p[:, 2] == 0)
    assert p[:, 0].max() > p0[:, 0].max() + 0.2        # the column collapsed and spread
    assert p[:, 1].mean() < p0[:, 1].mean()            # and its centre of mass fell
