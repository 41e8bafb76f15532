"""The oracle's restatement of FluidSolver2D.cu (the reference's own 2D step)
against hand-computed cases, one per quirk of that step.

The reference has no tests or golden outputs for its 2D solver, so each phase
is pinned here by values worked out from the reference's expressions
(FluidSolver2D.cu and utility.cu line numbers in each test), in float32.
"""
import numpy as np
import pytest

f32 = np.float32
VU = f32(-2.0 ** 31)


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    return oracle


def _box(W=6, H=5):
    lab = np.full((H, W), 2, np.uint8)
    lab[0] = lab[-1] = 0
    lab[:, 0] = lab[:, -1] = 0
    return lab


def _hat(r):
    a = abs(f32(r))
    return f32(1) - a if float(a - f32(1)) <= 1e-8 else f32(0)


def test_p2g_weights_by_cell_centre(O):
    """accumulateDenAndNum (:259-274): u and v faces (i, j) both use the
    centre ((i + .5) dx, (j + .5) dx); applyNumDen (:276-288) leaves 0 where
    the weight sum is 0.  Two particles: a weighted mean in particle order."""
    W, H, dx = 6, 5, f32(0.25)
    r = O.Ref2D(W, H, dx, 0.01)
    r.set_labels(_box(W, H))
    pos = np.array([[0.70, 0.40, 0], [0.80, 0.55, 0]], np.float32)
    vel = np.array([[1.5, -2.0, 0], [-0.5, 3.0, 0]], np.float32)
    r.set_particles(pos, vel)
    r.phase(O.PH_P2G)
    u = r.grid(O.GRID_U).reshape(H, W + 1)
    v = r.grid(O.GRID_V).reshape(H + 1, W)
    nz = 0
    for j in range(H + 1):
        for i in range(W + 1):
            c = [(f32(i) + f32(0.5)) * dx, (f32(j) + f32(0.5)) * dx]
            k = [_hat((p[0] - c[0]) / dx) * _hat((p[1] - c[1]) / dx) for p in pos]
            den = f32(0) + k[0] + k[1]
            nu = f32(0) + vel[0, 0] * k[0] + vel[1, 0] * k[1]
            nv = f32(0) + vel[0, 1] * k[0] + vel[1, 1] * k[1]
            nz += den != 0
            if j < H:
                assert u[j, i] == (nu / den if den != 0 else 0), (i, j)
            if i < W:
                assert v[j, i] == (nv / den if den != 0 else 0), (i, j)
    assert nz == 4  # both particles' hats cover the same 2 x 2 face centres


def test_forces_skip_unknown_faces(O):
    """applyForces (:362-381): gravity dt * -9.81 on v faces that are not
    VEL_UNKNOWN; u gets dt * 0."""
    W, H = 4, 4
    r = O.Ref2D(W, H, 0.25, 0.01)
    r.set_labels(_box(W, H))
    v = np.arange(W * (H + 1), dtype=np.float64)
    v[3] = VU
    r.set_grid(O.GRID_V, v)
    r.phase(O.PH_FORCES)
    out = r.grid(O.GRID_V)
    g = f32(0.01) * f32(-9.81)
    exp = (v.astype(np.float32) + g).astype(np.float64)
    exp[3] = VU
    assert np.array_equal(out, exp)


def test_projection_quirks(O):
    """applyPressure (:720-757): a face with a FLUID side and a SOLID side is
    0, a FLUID/FLUID or FLUID/AIR face gets the pressure gradient, a face with
    no FLUID side becomes VEL_UNKNOWN, the border faces i = 0, i = W (u) and
    j = 0, j = H (v) keep their values."""
    W, H, dx, dt = 5, 4, f32(0.2), f32(0.01)
    lab = _box(W, H)
    lab[1, 1] = lab[1, 2] = 1  # FLUID at (1,1), (2,1); AIR elsewhere inside
    r = O.Ref2D(W, H, dx, dt)
    r.set_labels(lab)
    rng = np.random.default_rng(0)
    u0 = rng.standard_normal((W + 1) * H).astype(np.float32).astype(np.float64)
    v0 = rng.standard_normal(W * (H + 1)).astype(np.float32).astype(np.float64)
    p = np.zeros(W * H)
    p[1 * W + 1], p[1 * W + 2] = 3.0, 5.0
    r.set_grid(O.GRID_U, u0); r.set_grid(O.GRID_V, v0); r.set_grid(O.GRID_P, p)
    r.phase(O.PH_PROJECT)
    u = r.grid(O.GRID_U).reshape(H, W + 1)
    v = r.grid(O.GRID_V).reshape(H + 1, W)
    U0 = u0.reshape(H, W + 1); V0 = v0.reshape(H + 1, W)
    scale = dt / (f32(1000) * dx)
    assert u[1, 1] == 0.0                                  # SOLID | FLUID
    assert u[1, 2] == f32(f32(U0[1, 2]) - scale * (f32(5) - f32(3)))   # FLUID | FLUID
    assert u[1, 3] == f32(f32(U0[1, 3]) - scale * (f32(0) - f32(5)))   # FLUID | AIR
    assert u[2, 2] == VU and u[1, 4] == VU                # AIR | AIR
    assert np.array_equal(u[:, 0], U0[:, 0]) and np.array_equal(u[:, W], U0[:, W])
    assert v[1, 1] == 0.0 and v[2, 1] == f32(f32(V0[2, 1]) - scale * (f32(0) - f32(3)))
    assert v[3, 3] == VU
    assert np.array_equal(v[0], V0[0]) and np.array_equal(v[H], V0[H])


def test_g2p_is_1d_linear_in_the_cell(O):
    """interpVel (:792-820): u is linear in x between the cell's two u faces
    (independent of y), v linear in y; outside the grid both are VEL_UNKNOWN.
    gridToParticles (:822-853) blends alpha * PIC + (1 - alpha) * FLIP."""
    W, H, dx = 4, 4, f32(0.25)
    r = O.Ref2D(W, H, dx, 0.01, pic_weight=0.25)
    r.set_labels(_box(W, H))
    u = np.arange((W + 1) * H, dtype=np.float32).astype(np.float64)
    v = (10 + np.arange(W * (H + 1))).astype(np.float32).astype(np.float64)
    r.set_grid(O.GRID_U, u); r.set_grid(O.GRID_V, v)
    r.set_grid(O.GRID_US, u - 1); r.set_grid(O.GRID_VS, v - 2)
    pos = np.array([[0.3, 0.6, 0], [1.2, 0.1, 0]], np.float32)
    vel = np.array([[0.5, 0.25, 0], [0, 0, 0]], np.float32)
    r.set_particles(pos, vel)
    r.phase(O.PH_G2P)
    _, vo = r.particles()
    i, j = 1, 2
    cx, cy = (f32(i) + f32(.5)) * dx, (f32(j) + f32(.5)) * dx
    off = dx / f32(2)
    x1, x2, y1, y2 = cx - off, cx + off, cy - off, cy + off
    U = u.reshape(H, W + 1).astype(np.float32); V = v.reshape(H + 1, W).astype(np.float32)
    pu = ((x2 - pos[0, 0]) / (x2 - x1)) * U[j, i] + ((pos[0, 0] - x1) / (x2 - x1)) * U[j, i + 1]
    pv = ((y2 - pos[0, 1]) / (y2 - y1)) * V[j, i] + ((pos[0, 1] - y1) / (y2 - y1)) * V[j + 1, i]
    fu = ((x2 - pos[0, 0]) / (x2 - x1)) * f32(1) + ((pos[0, 0] - x1) / (x2 - x1)) * f32(1)
    fv = ((y2 - pos[0, 1]) / (y2 - y1)) * f32(2) + ((pos[0, 1] - y1) / (y2 - y1)) * f32(2)
    a = f32(0.25)
    assert vo[0, 0] == pu * a + (vel[0, 0] + fu) * (f32(1) - a)
    assert vo[0, 1] == pv * a + (vel[0, 1] + fv) * (f32(1) - a)
    # a particle beyond x = W dx interpolates VEL_UNKNOWN for both PIC and FLIP
    r.set_particles(np.array([[1.1, 0.5, 0]], np.float32), np.array([[1.0, 1.0, 0]], np.float32))
    r.phase(O.PH_G2P)
    _, vo = r.particles()
    assert vo[0, 0] == VU * a + (f32(1) + VU) * (f32(1) - a)


def test_advection_moves_into_solid_neighbour(O):
    """advectParticles (:1122-1166) with C = 1: a particle that lands in a
    SOLID cell goes to the nearest SOLID cell centre of its 8 neighbours
    (projectParticle, :1072-1119 -- the reference picks SOLID first)."""
    W, H, dx, dt = 6, 6, f32(0.25), f32(0.1)
    lab = _box(W, H)
    lab[1:5, 1:5] = 1
    r = O.Ref2D(W, H, dx, dt)
    r.set_labels(lab)
    u = np.full((W + 1) * H, -1.0)      # everything moves left at 1 m/s
    r.set_grid(O.GRID_U, u); r.set_grid(O.GRID_V, np.zeros(W * (H + 1)))
    r.set_particles(np.array([[0.26, 0.9, 0]], np.float32), np.zeros((1, 3), np.float32))
    r.phase(O.PH_ADVECT)
    po, _ = r.particles()
    # dT = C dx / (|v| + FLT_MIN) = 0.25 >= dt: one substep of 0.1 to x = 0.16,
    # in SOLID cell (0, 3); its SOLID neighbours are (0, 4) and (0, 2) (column
    # -1 is outside, column 1 is FLUID), and (0, 4) is the nearer
    x, y = f32(0.26) + f32(-1) * f32(0.1), f32(0.9)
    cands = [(0, 4), (0, 2)]
    d = [np.hypot(float((f32(a) + f32(.5)) * dx - x), float((f32(c) + f32(.5)) * dx - y)) for a, c in cands]
    a, c = cands[int(np.argmin(d))]
    assert (a, c) == (0, 4)
    assert po[0, 0] == x + ((f32(a) + f32(.5)) * dx - x)
    assert po[0, 1] == y + ((f32(c) + f32(.5)) * dx - y)


def test_cleanup_deletes_in_order(O):
    """cleanUpParticles (:1171-1204): out-of-grid and NaN particles are
    erased, the others keep their order; (int) truncation keeps a particle
    at x in (-dx, 0) in column 0."""
    W, H, dx = 4, 4, f32(0.25)
    lab = _box(W, H)
    lab[1:3, 1:3] = 1
    r = O.Ref2D(W, H, dx, 0.01)
    r.set_labels(lab)
    pos = np.array([[0.4, 0.4, 0], [-0.3, 0.5, 0], [0.6, 0.6, 0], [1.2, 0.5, 0], [-0.1, 0.4, 0]], np.float32)
    vel = np.arange(15, dtype=np.float32).reshape(5, 3)
    r.set_particles(pos, vel)
    r.phase(O.PH_CLEANUP)
    po, vo = r.particles()
    assert len(po) == 3 and r.stats()["removed"] == 2
    assert np.array_equal(vo[:2, :2], vel[[0, 2], :2])
    # the last one sits in SOLID cell (0, 1); its nearest SOLID neighbour is
    # (0, 2), and the move is pos + 1 * (centre - pos), not the centre itself
    x, y = f32(-0.1), f32(0.4)
    cx, cy = (f32(0) + f32(.5)) * dx, (f32(2) + f32(.5)) * dx
    assert po[2, 0] == x + f32(1) * (cx - x) and po[2, 1] == y + f32(1) * (cy - y)


def test_pressure_matches_a_direct_solve(O):
    """pressureSolve (:566-718): RHS and 5-point operator of constructRHS /
    constructA, solved exactly (numpy dense solve standing in for cuDSS)."""
    W, H, dx, dt = 7, 6, f32(1 / 7), f32(0.01)
    lab = _box(W, H)
    lab[1:3, 1:6] = 1
    lab[3, 2:4] = 1
    r = O.Ref2D(W, H, dx, dt, tol=1e-13)
    r.set_labels(lab)
    rng = np.random.default_rng(3)
    u = rng.standard_normal((W + 1) * H).astype(np.float32)
    v = rng.standard_normal(W * (H + 1)).astype(np.float32)
    r.set_grid(O.GRID_U, u); r.set_grid(O.GRID_V, v)
    assert r.phase(O.PH_PRESSURE) == 0
    p = r.grid(O.GRID_P).reshape(H, W)
    U = u.reshape(H, W + 1); V = v.reshape(H + 1, W)
    cells = [(i, j) for j in range(H) for i in range(W) if lab[j, i] == 1]
    num = {c: n for n, c in enumerate(cells)}
    A = np.zeros((len(cells), len(cells)))
    b = np.zeros(len(cells))
    scale = (f32(1000) * dx) / dt
    for n, (i, j) in enumerate(cells):
        rr = -scale * (U[j, i + 1] - U[j, i] + V[j + 1, i] - V[j, i])
        if lab[j, i - 1] == 0: rr -= scale * (U[j, i] - f32(0))
        if lab[j, i + 1] == 0: rr += scale * (U[j, i + 1] - f32(0))
        if lab[j - 1, i] == 0: rr -= scale * (V[j, i] - f32(0))
        if lab[j + 1, i] == 0: rr += scale * (V[j + 1, i] - f32(0))
        b[n] = rr
        for (a, c) in ((i - 1, j), (i + 1, j), (i, j - 1), (i, j + 1)):
            if lab[c, a] in (1, 2):
                A[n, n] += 1
            if lab[c, a] == 1:
                A[n, num[(a, c)]] = -1
    x = np.linalg.solve(A, b)
    got = np.array([p[j, i] for (i, j) in cells])
    assert np.allclose(got, x.astype(np.float32), rtol=1e-5, atol=1e-5 * np.abs(x).max())
    assert np.all(p[lab != 1] == 0)


def test_dam_break_runs_and_keeps_particles(O):
    """Config-1 scene under the reference's 2D step for 30 steps: finite,
    nothing deleted from a closed box, the column falls."""
    from fluidprjct_b200 import scenes
    lab = scenes.dam_break_2d(32)
    pos = O.seed2d(lab, 1 / 32, 4, 0)
    r = O.Ref2D(32, 32, 1 / 32, 0.005, pic_weight=0.05, tol=1e-10)
    r.set_labels(lab)
    r.set_particles(pos)
    y0 = pos[:, 1].mean()
    assert r.step(30) == 0
    po, vo = r.particles()
    assert np.isfinite(po).all() and np.isfinite(vo).all()
    assert len(po) == len(pos)
    assert po[:, 1].mean() < y0


def test_extrapolation_waves_and_stride_quirk(O):
    """extrapolateGridFluidData (:1207-1295), enabled in the G2P -> advection
    gap: a VEL_UNKNOWN face next to known faces becomes the mean of its known
    8-neighbours (wave 1), the next ring the mean of older waves (wave 2).
    The initial front of the u grid reads markers at stride W, not W + 1
    (checkNeighbors, :1049-1066)."""
    W, H = 6, 5
    r = O.Ref2D(W, H, 0.2, 0.01)
    r.set_extrapolate(True)
    lab = _box(W, H)
    r.set_labels(lab)
    r.set_particles(np.zeros((0, 3), np.float32))
    v = np.full((H + 1, W), VU, np.float64)
    v[0, :3] = [1.0, 2.0, 4.0]                     # known values in the bottom row
    r.set_grid(O.GRID_V, v)
    u = np.full((H, W + 1), VU, np.float64)
    u[1, 0] = 8.0                                  # one known u face, (i, j) = (0, 1): true index 7
    r.set_grid(O.GRID_U, u)
    r.phase(O.PH_ADVECT)
    uo = r.grid(O.GRID_U).reshape(H, W + 1)
    # The first front tests markers at a + b*W = 7, i.e. cell (1, 1): the
    # neighbours of (1, 1) join wave 1.  (0, 0) and (0, 2) are true neighbours
    # of the known face and take its value; (2, 0..2) have no older neighbour
    # and become 0/0 = NaN, as in the reference; (1, 1) itself is not in wave 1.
    assert uo[0, 0] == 8.0 and uo[2, 0] == 8.0
    assert np.isnan(uo[0, 2]) and np.isnan(uo[1, 2]) and np.isnan(uo[2, 2])
