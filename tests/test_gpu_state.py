"""Per-step log and exact-resume snapshots on the GPU.

fp_set_step_log writes one JSON line per step (the reference prints its
frameStep phase timers once, at the end of run(), FluidSolver3D.cu:3149-3162).
fp_save_state / fp_load_state snapshot everything a step depends on: grids,
labels, particles, the body and the previous pressure that warm-starts the
solve.  A resumed run matches the uninterrupted one up to the order of P2G's
shared-memory sums (relative L2 1e-5, as the phase parity bar).
"""
import json

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _pool(O, **kw):
    from fluidprjct_b200 import capi, scenes
    n = 32
    cfg = dict(dx=1.0 / n, dt=0.003, pic_weight=0.05, solver="pcg_mg", tol=1e-7, body_radius=0.1,
               body_density=0.6, body_pos=(0.45, 0.62, 0.5), active_body=1, advection="rk2", collision="sdf",
               output_format=capi.OUT_NONE)
    cfg.update(kw)
    s = capi.Solver(**cfg)
    lab = scenes.box_3d(n, n, n, 1.0 / n, 2.0, 0.55, 2.0)
    s.set_labels(lab)
    s.load_sdf(None)
    s.seed_particles(8, 3)
    return s, cfg, lab


def test_step_log_has_one_json_line_per_step(O, tmp_path):
    s, _, _ = _pool(O)
    log = tmp_path / "steps.jsonl"
    s.set_step_log(log)
    s.step(3)
    s.run(2)  # 2 * iter_per_frame + 1 steps
    s.set_step_log(None)
    s.step(1)  # not logged
    rows = [json.loads(line) for line in log.read_text().splitlines()]
    assert [r["step"] for r in rows] == [1, 2, 3, 4, 5, 6]
    for r in rows:
        assert r["solve_status"] == 0 and r["residual"] <= 1e-7 and r["particles"] > 0
        assert r["t_total"] > 0 and r["t_pressure"] > 0 and r["fluid_cells"] > 0
    assert rows[-1]["body_pos"][1] != rows[0]["body_pos"][1]
    s.close()


def test_state_snapshot_resumes_the_run(O, tmp_path):
    from fluidprjct_b200 import capi
    a, cfg, lab = _pool(O)
    a.step(4)
    snap = tmp_path / "state.bin"
    a.save_state(snap)
    a.step(4)
    b = capi.Solver(**cfg)
    b.load_state(snap)
    assert b.stats()["step"] == 4 and b.num_particles == a.num_particles
    b.step(4)
    sa, sb = a.stats(), b.stats()
    assert sa["step"] == sb["step"] == 8
    assert np.array_equal(a.labels(), b.labels())
    for g in (capi.GRID_U, capi.GRID_V, capi.GRID_W, capi.GRID_P):
        assert rel_l2(b.grid(g), a.grid(g)) <= 1e-5, g
    pa, va = a.particles()
    pb, vb = b.particles()
    assert rel_l2(pb, pa) <= 1e-6 and rel_l2(vb, va) <= 1e-5
    assert np.allclose(sb["body_pos"], sa["body_pos"], atol=1e-7)
    assert np.allclose(sb["body_vel"], sa["body_vel"], rtol=1e-4, atol=1e-7)
    assert abs(sb["pcg_iters"] - sa["pcg_iters"]) <= 1  # the warm start came along
    # a solver with another dt, a truncated file and a foreign file are refused
    c = capi.Solver(**dict(cfg, dt=0.004))
    with pytest.raises(capi.FluidError) as e:
        c.load_state(snap)
    assert e.value.code == capi.FP_ERR_ARG
    raw = snap.read_bytes()
    (tmp_path / "short.bin").write_bytes(raw[: len(raw) // 2])
    (tmp_path / "foreign.bin").write_bytes(b"not a state file at all")
    for bad in ("short.bin", "foreign.bin", "missing.bin"):
        with pytest.raises(capi.FluidError) as e:
            b.load_state(tmp_path / bad)
        assert e.value.code == capi.FP_ERR_IO
    for x in (a, b, c):
        x.close()
