"""Scene generation and the wave paddle on the GPU.

Level-set labels are checked against a label file the reference's own
DistrGen code wrote; seabed labels against the Python generator (same noise,
same bits); the paddle against the oracle; and the large seabed
configuration (256x128x256, paddle amplitude 0.05, period 1 s, dt = 0.001)
runs at full size.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu


def test_levelset_labels_on_gpu():
    from fluidprjct_b200 import capi
    ls = os.path.join(GOLDEN, "levelsets")
    solid = capi.read_levelset_file(os.path.join(ls, "solid_init.txt"))
    fluid = capi.read_levelset_file(os.path.join(ls, "fluid_init_ball.txt"))
    s = capi.Solver(dim=2, dx=1 / 40, dt=0.005, output_format=capi.OUT_NONE)
    s.set_labels_from_levelsets(solid, fluid)
    s2 = capi.Solver(dim=2, dx=1 / 40, dt=0.005, output_format=capi.OUT_NONE)
    s2.load_labels(os.path.join(ls, "labels_simple.txt"))
    assert np.array_equal(s.labels(), s2.labels())
    s.seed_particles(4, 0)
    assert s.num_particles == 4 * int((s.labels() == 1).sum())


@pytest.mark.parametrize("dims", [(64, 32, 48), (256, 128, 256)])
def test_seabed_labels_bit_exact(dims):
    from fluidprjct_b200 import capi, scenes
    W, H, D = dims
    dx = 1 / 128 if W == 256 else 1 / 32
    s = capi.Solver(dx=dx, dt=0.001, output_format=capi.OUT_NONE)
    s.scene_seabed(W, H, D, level=0.45, bed_base=0.15, bed_amp=0.05, seed=4, water_xmin=0.1)
    ref = scenes.seabed(W, H, D, dx, level=0.45, seed=4, water_xmin=0.1)
    assert np.array_equal(s.labels(), ref)


def _tank(O, n=32, dt=0.004, x_rest=0.15, amp=0.05, period=0.4):
    from fluidprjct_b200 import capi, scenes
    dx = 1.0 / n
    lab = scenes.box_3d(n, n, n, dx, 2.0, 0.5, 2.0, xmin=x_rest)
    s = capi.Solver(dx=dx, dt=dt, pic_weight=0.05, solver="pcg_mixed", tol=1e-9, output_format=capi.OUT_NONE)
    s.set_labels(lab)
    s.set_paddle(x_rest, amp, period)
    pos = O.seed3d(lab, dx, 8, 7)
    s.set_particles(pos)
    o = O.Sim3(n, n, n, dx, dt, fp64=False, pic_weight=0.05, tol=1e-12)
    o.set_labels(lab)
    o.set_paddle(x_rest, amp, period)
    o.set_particles(pos)
    return s, o, lab


def test_paddle_marking_and_steps_match_oracle(O):
    from fluidprjct_b200 import capi
    s, o, lab = _tank(O)
    s.phase(capi.PHASE_LABEL)
    o.phase(O.PH_LABEL)
    assert np.array_equal(s.labels(), o.labels()) and int((s.labels() == 3).sum()) > 0
    s.step(4)
    o.step(4)
    st = s.stats()
    ob = o.body_state()
    assert np.allclose(st["body_pos"][0], ob["pos"][0], rtol=0, atol=1e-12)
    assert np.allclose(st["body_vel"][0], ob["vel"][0], rtol=0, atol=1e-12)
    assert np.array_equal(s.labels(), o.labels())
    for g, go in ((capi.GRID_U, O.GRID_U), (capi.GRID_V, O.GRID_V), (capi.GRID_P, O.GRID_P)):
        assert rel_l2(s.grid(g), o.grid(go)) < 1e-4
    # the paddle pushes the water: positive x load on it as it moves in
    assert st["body_force"][0] < 0.0 < st["body_vel"][0]


def test_seabed_paddle_configuration():
    """The large seabed scene at full size: 256x128x256 (dx = 1/128), bed
    0.15 + 0.05 noise (seed 4), water to y < 0.45 behind a paddle at rest at
    x = 0.1 (amplitude 0.05, period 1 s), 8 ppc, dt = 0.001.  After a quarter
    period the paddle has pushed a crest above the still level next to it.
    On that step's pressure system the learned + MG, mixed and MG solves reach
    1e-6 faster than the plain PCG."""
    from fluidprjct_b200 import capi, learned
    s = capi.Solver(dx=1 / 128, dt=0.001, pic_weight=0.05, solver="pcg_mg", tol=1e-6, advection="rk2",
                    output_format=capi.OUT_NONE)
    s.scene_seabed(256, 128, 256, level=0.45, bed_base=0.15, bed_amp=0.05, seed=4, water_xmin=0.1)
    s.set_paddle(0.1, 0.05, 1.0)
    s.seed_particles(8, 4)
    n0 = s.num_particles
    assert n0 > 15_000_000
    s.step(250)
    st = s.stats()
    assert st["solve_status"] == 0 and st["residual"] <= 1e-6 and s.num_particles == n0
    assert abs(st["body_pos"][0] - (0.1 + 0.05)) < 1e-3  # a quarter period: full stroke
    p, _ = s.particles()
    assert np.isfinite(p).all()
    near = p[:, 0] < 0.3
    assert p[near, 1].max() > 0.45 + 2 / 128
    lab = s.labels()
    rhs = s.grid(capi.GRID_RHS)
    r = learned.compare_solvers(lab, rhs, learned.DEFAULT_WEIGHTS, repeats=1,
                                names=("pcg", "pcg_mixed", "pcg_mg", "pcg_learned"))
    print(n0, st["t_total"], r)
    for v in r.values():
        assert v["status"] == 0 and v["residual"] <= 1e-6
    for name in ("pcg_mixed", "pcg_mg", "pcg_learned"):
        assert r[name]["ms"] < r["pcg"]["ms"]
