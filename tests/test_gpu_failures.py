"""Failure paths of the step on the GPU, made to happen without any fault.

The persistent pressure solvers wait at grid barriers with a bounded number
of polls.  ``fp_set_wait_limit`` lowers that bound to a single poll, so a
block that is not the last to arrive gives up at once: the kernel records
DEV_TIMEOUT and every block returns at its next barrier.  Nothing waits on a
flag that no one sets, nothing traps, and every access stays in bounds.

Checked through the C ABI, for the solvers with a grid barrier:
  * the step returns FP_ERR_TIMEOUT;
  * the particles (positions and velocities) and the rigid body's state are
    those from before the step: the projection and G2P/advection kernels read
    the solve's status and skip, and the body is not integrated;
  * the next step with the default limit solves to tolerance and matches a
    fresh solver's first step from the same state (the host restored the
    solver's zero-state work grids after the timeout).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _pool_with_sphere(O, solver, n=40):
    from fluidprjct_b200 import capi, scenes
    dx = 1.0 / n
    lab = scenes.box_3d(n, n, n, dx, 2.0, 0.6, 2.0)
    kw = dict(dx=dx, dt=0.002, pic_weight=0.05, solver=solver, tol=1e-7, body_radius=0.1, body_density=0.5,
              body_pos=(0.5, 0.55, 0.5), active_body=1, advection="rk2")
    s = capi.Solver(**kw)
    s.set_labels(lab)
    s.load_sdf(None)
    lab2 = lab.copy()
    lab2[s.labels() == capi.BODY] = capi.BODY
    pos = O.seed3d(lab2, dx, 8, 5)
    vel = np.random.default_rng(5).uniform(-0.3, 0.3, pos.shape).astype(np.float32)
    s.set_particles(pos, vel)
    return s, kw, lab, pos, vel


@pytest.mark.parametrize("solver", ["pcg_mg", "pcg", "pcg_mixed"])
def test_timed_out_solve_changes_nothing_and_the_next_step_recovers(O, solver):
    from fluidprjct_b200 import capi
    s, kw, lab, pos, vel = _pool_with_sphere(O, solver)
    body0 = {k: list(s.stats()[k]) for k in ("body_pos", "body_vel", "body_omega")}

    s.set_wait_limit(1)
    with pytest.raises(capi.FluidError) as e:
        s.step(1)
    assert e.value.code == capi.FP_ERR_TIMEOUT
    st = s.stats()
    assert st["solve_status"] == capi.FP_ERR_TIMEOUT
    p1, v1 = s.particles()
    assert np.array_equal(p1, pos) and np.array_equal(v1, vel), "a timed-out step moved particles"
    for k, v in body0.items():
        assert st[k] == v, f"a timed-out step changed the body's {k}"

    # default limit again: the step solves, and equals a fresh solver's step
    s.set_wait_limit(0)
    s.step(1)
    st = s.stats()
    assert st["solve_status"] == capi.FP_OK and st["residual"] <= 1e-7, st
    f = capi.Solver(**kw)
    f.set_labels(lab)
    f.load_sdf(None)
    f.set_particles(pos, vel)
    f.step(1)
    assert np.array_equal(s.labels(), f.labels())
    for g in (capi.GRID_P, capi.GRID_U, capi.GRID_V, capi.GRID_W):
        assert rel_l2(s.grid(g), f.grid(g)) < 1e-5, g
    pa, va = s.particles()
    pb, vb = f.particles()
    assert rel_l2(pa, pb) < 1e-6 and rel_l2(va, vb) < 1e-5
    assert np.allclose(s.stats()["body_pos"], f.stats()["body_pos"], atol=1e-9)
    f.close()
    s.close()


def test_wait_limit_rejects_negative_values():
    from fluidprjct_b200 import capi
    s = capi.Solver(dx=0.05, dt=0.002)
    with pytest.raises(capi.FluidError) as e:
        s.set_wait_limit(-1)
    assert e.value.code == capi.FP_ERR_ARG
    s.close()
