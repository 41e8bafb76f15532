"""The oracle's SDF collision projection on the CPU (the checker of the GPU's
collision = sdf mode): with zero grid velocities, advection only projects,
so particles placed inside the sphere or behind the paddle face end exactly
dx/4 outside, along the normal, and particles outside do not move."""
import numpy as np


def _sim(O, n=20):
    dx = 1.0 / n
    lab = np.full((n, n, n), 2, np.uint8)
    lab[0], lab[-1], lab[:, 0], lab[:, -1], lab[:, :, 0], lab[:, :, -1] = 0, 0, 0, 0, 0, 0
    o = O.Sim3(n, n, n, dx, 0.002, fp64=True, rk2=True)
    o.set_labels(lab)
    return o, dx


def test_sphere_push_out(O):
    o, dx = _sim(O)
    c, r = np.array([0.5, 0.5, 0.5]), 0.2
    o.set_sphere(c, r, 1.0)
    o.set_collision(True)
    rng = np.random.default_rng(1)
    d = rng.normal(size=(500, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rad = rng.uniform(0.02, 0.35, 500)
    pos = (c + d * rad[:, None]).astype(np.float32)
    o.set_particles(pos)
    o.phase(O.PH_ADVECT)
    p, _ = o.particles()
    r32 = float(np.float32(r))
    inside = rad < r32 + 0.25 * dx
    phi = np.linalg.norm(p - c, axis=1) - r32
    assert np.allclose(phi[inside], 0.25 * dx, atol=1e-6)
    # moved radially: the direction from the centre is kept
    dd = (p[inside] - c) / np.linalg.norm(p[inside] - c, axis=1, keepdims=True)
    assert np.allclose(dd, d[inside], atol=1e-5)
    assert np.allclose(p[~inside], pos[~inside], atol=1e-6)


def test_paddle_push_out(O):
    o, dx = _sim(O)
    o.set_paddle(0.3, 0.0, 1.0)
    o.set_collision(True)
    pos = np.array([[0.1, 0.5, 0.5], [0.29, 0.4, 0.6], [0.5, 0.5, 0.5]], np.float32)
    o.set_particles(pos)
    o.phase(O.PH_ADVECT)
    p, _ = o.particles()
    assert np.allclose(p[:2, 0], 0.3 + 0.25 * dx, atol=1e-6)
    assert np.allclose(p[:2, 1:], pos[:2, 1:], atol=1e-7)
    assert np.allclose(p[2], pos[2], atol=1e-7)
