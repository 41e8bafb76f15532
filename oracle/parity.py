"""Phase-by-phase parity of one step against the FP64 oracle, at any size.

TEST INFRASTRUCTURE ONLY (the checker): used by ``tests/`` and by
``bench.py``'s parity leg, never by the product package.  It drives the
product through its C ABI (``fluidprjct_b200.capi.Solver``) and the oracle
(``oracle.Sim3`` in FP64 mode) side by side on the same labels and
particles, and feeds every phase of the GPU step and of the oracle step the
same inputs -- the GPU's output of the phase before -- so that each error
belongs to one phase.  Phases follow ``frameStep`` (FluidSolver3D.cu:
3030-3098): label, P2G, save, forces, pressure, projection, body, G2P,
advection.

Errors are relative L2 norms ||gpu - oracle|| / ||oracle|| over the whole
array, the face-velocity components relative to the norm of the whole
velocity field (u, v, w together: a component that is zero up to rounding
in the oracle, like w of a dam break in its first step, has no meaningful
norm of its own); labels are compared for equality.  The GPU holds
positions and the pressure in FP32, so two FP32 floors are reported beside
the errors: positions are compared in units of the FP32 spacing (ulp) of the
oracle's coordinate, and the FP64 residual of the FP32-stored pressure has
the rounding floor ||A|| 2^-24 ||p|| / ||b|| with ||A|| <= 12 for the
7-point operator.  The pressure is compared with the
oracle's FP64 solve of its own right-hand side (Jacobi PCG to 1e-12, which
stands in for the reference's direct cuDSS solve) unless ``exact_solve`` is
False: then the GPU's pressure is checked only through its FP64 residual
||b - A p|| / ||b|| with the oracle's right-hand side and operator (cheap at
any size).
"""
from __future__ import annotations

import time

import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def vel_rel_l2(gpu_grids, or_grids):
    """Per-component errors relative to the norm of the whole velocity field."""
    den = np.sqrt(sum(float(np.sum(np.asarray(b, np.float64) ** 2)) for b in or_grids))
    den = den if den > 0 else 1.0
    return [float(np.linalg.norm(np.asarray(a, np.float64).ravel() - np.asarray(b, np.float64).ravel()) / den)
            for a, b in zip(gpu_grids, or_grids)]


def ulp_errors(p_gpu, p_or):
    """Per-particle largest coordinate error in FP32 ulps of the oracle's coordinate."""
    p_or = np.asarray(p_or, np.float64)
    ulp = np.spacing(np.abs(p_or).astype(np.float32)).astype(np.float64)
    return (np.abs(np.asarray(p_gpu, np.float64) - p_or) / np.maximum(ulp, np.spacing(np.float32(1e-30)))).max(axis=1)


def step_phases(s, o, dx, exact_solve=True, body_mass=None):
    """One step of solver ``s`` (capi.Solver) and oracle ``o`` (oracle.Sim3,
    fp64) phase by phase from identical inputs; returns a dict of errors and
    the oracle's wall time.  Both must hold the same labels and particles
    (and body) on entry; afterwards both hold the GPU's step.  body_mass:
    the sphere's mass when a body is coupled (its force is then compared)."""
    from fluidprjct_b200 import capi
    import oracle.oracle as O
    grids = ((capi.GRID_U, O.GRID_U), (capi.GRID_V, O.GRID_V), (capi.GRID_W, O.GRID_W))
    saved = ((capi.GRID_U_SAVED, O.GRID_US), (capi.GRID_V_SAVED, O.GRID_VS), (capi.GRID_W_SAVED, O.GRID_WS))
    res = {}
    t_or = 0.0

    def both(ph_s, ph_o):
        nonlocal t_or
        s.phase(ph_s)
        t0 = time.perf_counter()
        rc = o.phase(ph_o)
        t_or += time.perf_counter() - t0
        return rc

    def copy_to_oracle(pairs):
        for g, go in pairs:
            o.set_grid(go, s.grid(g).astype(np.float64))

    both(capi.PHASE_LABEL, O.PH_LABEL)
    res["labels_bitexact"] = bool(np.array_equal(s.labels(), o.labels()))
    both(capi.PHASE_P2G, O.PH_P2G)
    for name, e in zip("uvw", vel_rel_l2([s.grid(g) for g, _ in grids], [o.grid(go) for _, go in grids])):
        res[f"p2g_{name}_rel_l2"] = e
    both(capi.PHASE_SAVE, O.PH_SAVE)
    copy_to_oracle(grids + saved)
    both(capi.PHASE_FORCES, O.PH_FORCES)
    for name, e in zip("uvw", vel_rel_l2([s.grid(g) for g, _ in grids], [o.grid(go) for _, go in grids])):
        res[f"forces_{name}_rel_l2"] = e
    copy_to_oracle(grids)
    # pressure: the GPU solve of its system against the oracle's FP64 solve of its own
    s.phase(capi.PHASE_PRESSURE)
    st = s.stats()
    res["solve_residual"] = float(st["residual"])
    res["solve_iters"] = int(st["pcg_iters"])
    p_gpu = s.grid(capi.GRID_P).astype(np.float64).ravel()
    t0 = time.perf_counter()
    b = o.rhs()
    res["rhs_rel_l2"] = rel_l2(s.grid(capi.GRID_RHS), b)
    if exact_solve:
        o.phase(O.PH_PRESSURE)
        p_or = o.grid(O.GRID_P)
        res["p_rel_l2"] = rel_l2(p_gpu, p_or)
    ap = o.apply(p_gpu)
    fl = o.labels().ravel() == 1
    bn = max(np.linalg.norm(b[fl]), 1e-300)
    res["p_fp64_residual"] = float(np.linalg.norm((b - ap)[fl]) / bn)
    res["p_round_floor"] = float(12.0 * 2.0 ** -24 * np.linalg.norm(p_gpu[fl]) / bn)
    t_or += time.perf_counter() - t0
    o.set_grid(O.GRID_P, p_gpu)
    both(capi.PHASE_PROJECT, O.PH_PROJECT)
    for name, e in zip("uvw", vel_rel_l2([s.grid(g) for g, _ in grids], [o.grid(go) for _, go in grids])):
        res[f"project_{name}_rel_l2"] = e
    if body_mass is not None:
        # the face-fraction force of the same pressure (FP64 reductions on both
        # sides); the GPU's body_force also holds the weight m g
        f_or = o.body_force()
        s.phase(capi.PHASE_BODY)
        st = s.stats()
        weight = np.array([0.0, body_mass * float(np.float32(-9.81)), 0.0])
        f_gpu = np.array(st["body_force"]) - weight
        res["body_force_rel"] = rel_l2(f_gpu, f_or[:3])
        res["body_torque_abs_over_force"] = float(np.linalg.norm(np.array(st["body_torque"]) - f_or[3:])
                                                  / max(np.linalg.norm(f_or[:3]), 1e-300))
    copy_to_oracle(grids + saved)
    both(capi.PHASE_G2P, O.PH_G2P)
    _, v_gpu = s.particles()
    _, v_or = o.particles()
    res["g2p_vel_rel_l2"] = rel_l2(v_gpu, v_or)
    o.set_particles(*s.particles())
    both(capi.PHASE_ADVECT, O.PH_ADVECT)
    p_gpu, _ = s.particles()
    p_or, _ = o.particles()
    err = np.abs(p_gpu - p_or).max(axis=1)
    ulps = ulp_errors(p_gpu, p_or)
    res["advect_pos_rel_l2"] = rel_l2(p_gpu, p_or)
    res["advect_frac_within_8ulp"] = float(np.mean(ulps <= 8.0))
    res["advect_ulp_p999"] = float(np.quantile(ulps, 0.999)) if len(ulps) else 0.0
    res["advect_frac_within_1e-5dx"] = float(np.mean(err <= 1e-5 * dx))
    res["advect_max_err_dx"] = float(err.max() / dx) if len(err) else 0.0
    res["oracle_seconds"] = round(t_or, 2)
    return res


def full_step(s, o):
    """One whole step of both (each from the same state, each with its own
    solver); the errors of the GPU step's grids and particles against the
    FP64 oracle's step."""
    from fluidprjct_b200 import capi
    import oracle.oracle as O
    t0 = time.perf_counter()
    s.step(1)
    o.step(1)
    res = {"labels_bitexact": bool(np.array_equal(s.labels(), o.labels()))}
    pairs = ((capi.GRID_U, O.GRID_U), (capi.GRID_V, O.GRID_V), (capi.GRID_W, O.GRID_W))
    for name, e in zip("uvw", vel_rel_l2([s.grid(g) for g, _ in pairs], [o.grid(go) for _, go in pairs])):
        res[f"{name}_rel_l2"] = e
    res["p_rel_l2"] = rel_l2(s.grid(capi.GRID_P), o.grid(O.GRID_P))
    pg, vg = s.particles()
    po, vo = o.particles()
    res["vel_rel_l2"] = rel_l2(vg, vo)
    res["pos_rel_l2"] = rel_l2(pg, po)
    res["seconds"] = round(time.perf_counter() - t0, 2)
    return res
