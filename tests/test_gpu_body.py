"""Rigid-body coupling on the GPU against the oracle and against physics.

The body is an analytic sphere (the rigid-body drop configuration).  Marking
of BODY cells is bit-exact; the face-fraction pressure force equals the
oracle's FP64 evaluation on the same pressure; the force on a submerged body
in still water is its buoyancy.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _pool(O, n=40, level=0.7, c=(0.5, 0.35, 0.5), r=0.12, density=0.5, seed=3, dt=0.002, **kw):
    from fluidprjct_b200 import capi, scenes
    dx = 1.0 / n
    lab = scenes.box_3d(n, n, n, dx, 2.0, level, 2.0)
    s = capi.Solver(dx=dx, dt=dt, pic_weight=0.05, solver="pcg_mixed", tol=1e-9, body_radius=r,
                    body_density=density, body_pos=c, active_body=1, **kw)
    s.set_labels(lab)
    s.load_sdf(None)
    marked = s.labels()
    lab2 = lab.copy()
    lab2[marked == 3] = 3
    pos = O.seed3d(lab2, dx, 8, seed)
    s.set_particles(pos)
    r32 = float(np.float32(r))  # the library holds the radius as float32
    mass = float(np.float32(density)) * 1000.0 * 4.0 / 3.0 * np.pi * r32 ** 3
    o = O.Sim3(n, n, n, dx, dt, fp64=False, pic_weight=0.05, tol=1e-12)
    o.set_labels(lab)
    o.set_sphere(np.array(c, np.float64), r, mass)
    o.set_particles(pos)
    return s, o, lab, pos, mass


def test_body_marking_bit_exact(O):
    from fluidprjct_b200 import capi
    s, o, lab, pos, _ = _pool(O, n=48, c=(0.47, 0.41, 0.53), r=0.13)
    s.phase(capi.PHASE_LABEL)
    o.phase(O.PH_LABEL)
    assert np.array_equal(s.labels(), o.labels())
    assert int((s.labels() == 3).sum()) > 1000


def test_body_force_matches_oracle_and_buoyancy(O):
    from fluidprjct_b200 import capi
    s, o, lab, pos, mass = _pool(O, n=48)
    for ph_s, ph_o in ((capi.PHASE_LABEL, O.PH_LABEL), (capi.PHASE_P2G, O.PH_P2G), (capi.PHASE_SAVE, O.PH_SAVE),
                       (capi.PHASE_FORCES, O.PH_FORCES), (capi.PHASE_PRESSURE, O.PH_PRESSURE)):
        s.phase(ph_s)
        o.phase(ph_o)
    # same pressure on both sides -> the FP64 force reductions must agree
    o.set_grid(O.GRID_P, s.grid(capi.GRID_P).astype(np.float64))
    f_ref = o.body_force()
    s.phase(capi.PHASE_BODY)
    st = s.stats()
    g = float(np.float32(-9.81))  # the library's gravity constant is the float -9.81f
    f_gpu = np.array(st["body_force"]) - mass * np.array([0.0, g, 0.0])
    assert np.allclose(f_gpu, f_ref[:3], rtol=1e-9, atol=1e-9 * abs(f_ref[1]))
    assert np.allclose(np.array(st["body_torque"]), f_ref[3:], atol=1e-9 * abs(f_ref[1]))
    # buoyancy of the fully submerged sphere in still water (staircase error O(dx/r))
    V = 4.0 / 3.0 * np.pi * 0.12 ** 3
    assert 0.97 < f_gpu[1] / (1000 * 9.81 * V) < 1.12
    # integration: v = (F + m g)/m * dt from rest
    assert np.allclose(st["body_vel"][1], (f_gpu[1] + mass * g) / mass * float(np.float32(0.002)), rtol=1e-6)


def test_body_steps_match_oracle(O):
    from fluidprjct_b200 import capi
    s, o, lab, pos, mass = _pool(O, n=40, c=(0.5, 0.62, 0.5), r=0.1)
    s.step(3)
    o.step(3)
    st = s.stats()
    ob = o.body_state()
    assert np.allclose(st["body_pos"], ob["pos"], atol=1e-6)
    assert np.allclose(st["body_vel"], ob["vel"], rtol=1e-3, atol=1e-5)
    assert np.array_equal(s.labels(), o.labels())
    for g, go in ((capi.GRID_U, O.GRID_U), (capi.GRID_V, O.GRID_V), (capi.GRID_P, O.GRID_P)):
        assert rel_l2(s.grid(g), o.grid(go)) < 1e-4


def test_sdf_collision_matches_oracle(O):
    """collision = sdf: advected particles whose body SDF falls below dx/4 are
    projected along the sphere's normal to phi = dx/4 (and only SOLID cells
    keep the reference's label search).  From identical grids, G2P and
    advection agree with the oracle's restatement, no particle ends closer
    than dx/4 to the sphere, and the projection moved particles that the
    reference's label search leaves inside the body."""
    from fluidprjct_b200 import capi
    n, c, r = 40, (0.5, 0.45, 0.5), 0.1
    dx = 1.0 / n
    rng = np.random.default_rng(9)
    s, o, lab, pos, mass = _pool(O, n=n, c=c, r=r, density=2.0, collision="sdf")
    vel = rng.uniform(-0.5, 0.5, pos.shape).astype(np.float32)
    s.set_particles(pos, vel)
    o.set_particles(pos, vel)
    o.set_collision(True)
    s.phase(capi.PHASE_LABEL)
    o.phase(O.PH_LABEL)
    grids = {}
    for g, go in ((capi.GRID_U, O.GRID_U), (capi.GRID_V, O.GRID_V), (capi.GRID_W, O.GRID_W),
                  (capi.GRID_U_SAVED, O.GRID_US), (capi.GRID_V_SAVED, O.GRID_VS), (capi.GRID_W_SAVED, O.GRID_WS)):
        f = rng.uniform(-1, 1, s.grid_shape(g)).astype(np.float32)
        grids[g] = f
        s.set_grid(g, f)
        o.set_grid(go, f.astype(np.float64))
    for ph_s, ph_o in ((capi.PHASE_G2P, O.PH_G2P), (capi.PHASE_ADVECT, O.PH_ADVECT)):
        s.phase(ph_s)
        o.phase(ph_o)
    p_gpu, _ = s.particles()
    p_ref, _ = o.particles()
    err = np.abs(p_gpu - p_ref).max(axis=1)
    assert np.mean(err <= 1e-5 * dx) >= 0.999, np.sort(err)[-10:]
    r32 = float(np.float32(r))
    phi = np.linalg.norm(p_gpu.astype(np.float64) - np.array(c), axis=1) - r32
    assert phi.min() >= 0.25 * dx * (1 - 1e-4), phi.min()
    # the same advection with the reference's label search leaves particles inside
    t, _, _, _, _ = _pool(O, n=n, c=c, r=r, density=2.0)
    t.set_particles(pos, vel)
    t.phase(capi.PHASE_LABEL)
    for g, f in grids.items():
        t.set_grid(g, f)
    t.phase(capi.PHASE_G2P)
    t.phase(capi.PHASE_ADVECT)
    p_lab, _ = t.particles()
    phi_lab = np.linalg.norm(p_lab.astype(np.float64) - np.array(c), axis=1) - r32
    pushed = int((np.abs(p_gpu - p_lab).max(axis=1) > 1e-6).sum())
    assert pushed > 100 and int((phi_lab < 0).sum()) > 0, (pushed, int((phi_lab < 0).sum()))


def test_sdf_collision_full_steps_match_oracle(O):
    """Three coupled steps with collision = sdf against the oracle: labels
    bit-exact, grids within 1e-4 relative L2, and no particle inside the
    sphere at the end."""
    from fluidprjct_b200 import capi
    n, c, r = 40, (0.5, 0.5, 0.5), 0.1
    s, o, lab, pos, mass = _pool(O, n=n, c=c, r=r, density=2.0, collision="sdf")
    o.set_collision(True)
    s.step(3)
    o.step(3)
    assert np.array_equal(s.labels(), o.labels())
    for g, go in ((capi.GRID_U, O.GRID_U), (capi.GRID_V, O.GRID_V), (capi.GRID_P, O.GRID_P)):
        assert rel_l2(s.grid(g), o.grid(go)) < 1e-4
    st = s.stats()
    pg, _ = s.particles()
    com = np.array(st["body_pos"], np.float32).astype(np.float64)
    phi = np.linalg.norm(pg.astype(np.float64) - com, axis=1) - float(np.float32(r))
    assert phi.min() >= 0.25 / n * (1 - 1e-3), phi.min()


def test_rigid_body_drop_160(O):
    """Rigid-body drop at full size: 160^3, water y < 0.35 (8 ppc), sphere
    r = 0.12, density 0.5, released at (0.5, 0.7, 0.5) at rest."""
    from fluidprjct_b200 import capi, scenes
    n = 160
    lab = scenes.pool_3d(n, 0.35)
    s = capi.Solver(dx=1.0 / n, dt=0.002, pic_weight=0.05, solver="pcg_mixed", tol=1e-6, body_radius=0.12,
                    body_density=0.5, body_pos=(0.5, 0.7, 0.5), active_body=1, advection="rk2")
    s.set_labels(lab)
    s.load_sdf(None)
    s.seed_particles(8, 2)
    assert s.num_particles == 158 * 55 * 158 * 8
    s.step(5)
    st = s.stats()
    assert st["solve_status"] == 0 and st["residual"] <= 1e-6
    # in the air the body falls freely: v_y = -g t after 5 steps
    assert abs(st["body_vel"][1] - (-9.81 * 0.002 * 5)) < 1e-3
    assert abs(st["body_pos"][0] - 0.5) < 1e-6 and abs(st["body_pos"][2] - 0.5) < 1e-6


def test_pool_160_configuration():
    """The pool configuration at full size and length: 160^3, water y < 0.35,
    8 ppc (seed 2), sphere r = 0.12 at half the water's density released at
    (0.5, 0.7, 0.5), 300 steps of dt = 0.002 with the MG solver.  The sphere
    falls freely until its bottom meets the water (about 0.22 s), plunges and is
    pushed back up by the pressure; every solve converges and no particle is
    lost."""
    import time
    from fluidprjct_b200 import capi, scenes
    n = 160
    s = capi.Solver(dx=1.0 / n, dt=0.002, pic_weight=0.05, solver="pcg_mg", tol=1e-6, body_radius=0.12,
                    body_density=0.5, body_pos=(0.5, 0.7, 0.5), active_body=1, advection="rk2",
                    output_format=capi.OUT_NONE)
    s.set_labels(scenes.pool_3d(n, 0.35))
    s.load_sdf(None)
    s.seed_particles(8, 2)
    n0 = s.num_particles
    ys, vs, ms = [], [], []
    t0 = time.perf_counter()
    for _ in range(300):
        s.step(1)
        st = s.stats()
        assert st["solve_status"] == 0 and st["residual"] <= 1e-6
        ys.append(st["body_pos"][1])
        vs.append(st["body_vel"][1])
        ms.append(st["t_total"])
    wall = time.perf_counter() - t0
    print(f"pool 160^3: {n0} particles, {np.mean(ms[50:]):.3f} ms per step (device), {wall / 300 * 1e3:.3f} ms wall;"
          f" body y {ys[-1]:.4f}, lowest {min(ys):.4f}, v_y {vs[-1]:.4f}")
    assert s.num_particles == n0
    p, _ = s.particles()
    assert np.isfinite(p).all()
    k = int(np.argmin(ys))
    # plunged (centre below y = 0.35 + r) and rose again; the body stays inside the tank (the reference's
    # wall collisions are commented out, so nothing but the water stops it)
    assert 0.0 < min(ys) < 0.47 and k < 299 and max(vs[k:]) > 0.0


def _float_height(density, y0, n=64, steps=1500):
    from fluidprjct_b200 import capi, scenes
    s = capi.Solver(dx=1.0 / n, dt=0.002, pic_weight=0.05, solver="pcg_mg", tol=1e-6, body_radius=0.12,
                    body_density=density, body_pos=(0.5, y0, 0.5), active_body=1, advection="rk2",
                    output_format=capi.OUT_NONE)
    s.set_labels(scenes.pool_3d(n, 0.5))
    s.load_sdf(None)
    s.seed_particles(8, 2)
    ys = []
    for _ in range(steps):
        s.step(1)
        st = s.stats()
        assert st["solve_status"] == 0
        ys.append(st["body_pos"][1])
    return np.array(ys[-500:])


def test_sphere_floats_at_its_archimedes_depth():
    """The physical check of the face-fraction coupling: a sphere (r = 0.12)
    dropped from above a still pool (64^3, water to y = 0.5) settles where
    buoyancy balances its weight.  At half the water's density it floats half
    submerged (centre at the waterline, 0.5036 with the displaced water); at a
    quarter it floats a quarter submerged, its centre 0.042 higher (submerged
    cap height h with h^2 (3r - h) = r^3, h / 2r = 0.326).  The last 500 of
    1500 steps (3 s) stay within about a cell of those heights."""
    half = _float_height(0.5, 0.6)
    quarter = _float_height(0.25, 0.65)
    assert abs(half.mean() - 0.5036) < 0.02 and half.std() < 0.01
    assert abs((quarter.mean() - half.mean()) - 0.042) < 0.015 and quarter.std() < 0.01


def test_reference_body_forces_match_oracle(O):
    """body_forces = reference: the panel drag/lift of DragLiftForceCalculator
    (FluidSolver3D.cu:2674-2791) and the voxel buoyancy of applyBuoyancy
    (:2917-3026).  From the same labels, particles and (random) face
    velocities, the GPU force and torque match the oracle's."""
    from fluidprjct_b200 import capi
    s, o, lab, pos, mass = _pool(O, n=40, c=(0.5, 0.4, 0.5), r=0.12, body_forces="reference")
    o.set_reference_forces(True)
    s.phase(capi.PHASE_LABEL)
    o.phase(O.PH_LABEL)
    bv, om, c = [0.05, -0.2, 0.1], [0.0, 0.0, 0.0], [0.5, 0.4, 0.5]
    s.set_body_state(c, bv, om)
    o.set_body(np.array(bv), np.array(om), np.array(c))
    rng = np.random.default_rng(4)
    for g, go in ((capi.GRID_U, O.GRID_U), (capi.GRID_V, O.GRID_V), (capi.GRID_W, O.GRID_W)):
        f = rng.uniform(-1, 1, s.grid_shape(g)).astype(np.float32)
        s.set_grid(g, f)
        o.set_grid(go, f.astype(np.float64))
    s.phase(capi.PHASE_BODY)
    o.phase(O.PH_BODY)
    st = s.stats()
    ref = o.reference_forces()
    g = float(np.float32(-9.81))
    V = 4.0 / 3.0 * np.pi * float(np.float32(0.12)) ** 3
    # The voxels sample the sphere's volume.  The reference skips voxels with
    # 0 < sdf < cs although its fraction 1/2 - sdf/(2 cs) would count half of
    # them: about half a voxel shell (7.8 % of V here) is missing.  Only voxels
    # whose cell is FLUID (or holds a particle within 2 dx) count as
    # submerged, so a submerged body's interior (BODY cells, no particles)
    # does not: the reference's buoyancy is a surface shell's.
    assert 0.88 < ref[6] / V < 1.0 and 0.0 < ref[7] < 0.5 * ref[6]
    assert np.isfinite(ref).all() and abs(ref[0]) > 0
    f_ref = mass * np.array([0.0, g, 0.0]) + ref[:3] + np.array([0.0, 1000.0 * ref[7] * -g, 0.0])
    assert np.allclose(st["body_force"], f_ref, rtol=1e-5, atol=1e-5 * np.abs(ref[:3]).max())
    assert np.allclose(st["body_torque"], ref[3:6], rtol=1e-5, atol=1e-5 * np.abs(ref[3:6]).max())


def test_reference_lift_is_nan_where_the_reference_is(O):
    """The reference normalises n x u_rel for the lift (:2769-2771): a panel
    whose interpolated fluid velocity equals the body's (its stencil touches
    only faces set to the body velocity by the projection) gives 0/0, and the
    NaN survives the zero panel area.  A sphere at rest in still water hits
    that on its first step; the restatement does too, in the same place."""
    from fluidprjct_b200 import capi
    s, o, lab, pos, mass = _pool(O, n=40, c=(0.5, 0.4, 0.5), r=0.12, body_forces="reference")
    o.set_reference_forces(True)
    for ph_s, ph_o in ((capi.PHASE_LABEL, O.PH_LABEL), (capi.PHASE_P2G, O.PH_P2G), (capi.PHASE_SAVE, O.PH_SAVE),
                       (capi.PHASE_FORCES, O.PH_FORCES), (capi.PHASE_PRESSURE, O.PH_PRESSURE)):
        s.phase(ph_s)
        o.phase(ph_o)
    o.set_grid(O.GRID_P, s.grid(capi.GRID_P).astype(np.float64))
    s.phase(capi.PHASE_PROJECT)
    o.phase(O.PH_PROJECT)
    for g, go in ((capi.GRID_U, O.GRID_U), (capi.GRID_V, O.GRID_V), (capi.GRID_W, O.GRID_W)):
        o.set_grid(go, s.grid(g).astype(np.float64))
    s.phase(capi.PHASE_BODY)
    o.phase(O.PH_BODY)
    assert np.array_equal(np.isnan(s.stats()["body_force"]), np.isnan(o.body_state()["force"]))
    assert np.isnan(o.reference_forces()[:3]).any()


def test_run_writes_body_surface_points(O, tmp_path):
    """fp_run writes body_<frame>.ply beside the frames: the SDF voxel corners
    with |sdf| < dx/2 (generateSurfacePoints(0.5 dx), utility.cuh:339-374)."""
    from fluidprjct_b200 import capi
    s, o, lab, pos, mass = _pool(O, n=32, c=(0.5, 0.5, 0.5), r=0.15, output_format=capi.OUT_PLY_BINARY,
                                 output_template=str(tmp_path / "p_"), iter_per_frame=2)
    s.run(2)
    names = sorted(f.name for f in tmp_path.iterdir())
    assert names == ["body_0.ply", "body_1.ply", "body_2.ply", "csvRes.csv", "p_0.ply", "p_1.ply", "p_2.ply"]
    pts, _ = capi.read_ply_file(tmp_path / "body_2.ply")
    c = np.array(s.stats()["body_pos"])
    d = np.linalg.norm(pts - c, axis=1)
    assert len(pts) > 500 and np.all(np.abs(d - 0.15) < 0.5 / 32 + 1e-4)
