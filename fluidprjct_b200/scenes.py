"""Synthetic scenes of the benchmark configurations, as label grids.

Every scene has a one-cell SOLID wall around the domain (the precondition of
the reference's border reads) and marks as FLUID the cells whose centres lie
inside the water region.  Particles are then seeded by the native library
(``fp_seed_particles``, the reference's ``seedParticles`` with a fixed seed).
Label arrays have shape (D, H, W) (or (H, W) in 2D) with cell (i, j, k) at
``[k, j, i]``, the reference's ``i + j*W + k*W*H`` order.
"""
from __future__ import annotations

import numpy as np

SOLID, FLUID, AIR, BODY = 0, 1, 2, 3


def _walls(shape):
    lab = np.full(shape, AIR, np.uint8)
    if len(shape) == 3:
        lab[0, :, :] = lab[-1, :, :] = SOLID
        lab[:, 0, :] = lab[:, -1, :] = SOLID
        lab[:, :, 0] = lab[:, :, -1] = SOLID
    else:
        lab[0, :] = lab[-1, :] = SOLID
        lab[:, 0] = lab[:, -1] = SOLID
    return lab


def _centres(n, dx):
    return (np.arange(n, dtype=np.float64) + 0.5) * dx


def box_3d(W, H, D, dx, xmax, ymax, zmax, xmin=0.0, ymin=0.0, zmin=0.0):
    """Walls plus a FLUID box {xmin <= x < xmax, ...} of cell centres."""
    lab = _walls((D, H, W))
    x, y, z = _centres(W, dx), _centres(H, dx), _centres(D, dx)
    m = ((z >= zmin) & (z < zmax))[:, None, None] & ((y >= ymin) & (y < ymax))[None, :, None] & \
        ((x >= xmin) & (x < xmax))[None, None, :]
    lab[m & (lab != SOLID)] = FLUID
    return lab


def dam_break_3d(n=128, xmax=0.4, ymax=0.6, zmax=1.0):
    """Plain 3D dam break: n^3 grid, dx = 1/n, fluid box x<0.4, y<0.6, z<1."""
    return box_3d(n, n, n, 1.0 / n, xmax, ymax, zmax)


def dam_break_2d(n=64, xmax=0.4, ymax=0.5):
    """Plain 2D dam break: n^2 grid, dx = 1/n, fluid block x<0.4, y<0.5."""
    lab = _walls((n, n))
    dx = 1.0 / n
    x, y = _centres(n, dx), _centres(n, dx)
    m = (y < ymax)[:, None] & (x < xmax)[None, :]
    lab[m & (lab != SOLID)] = FLUID
    return lab


def pool_3d(n=160, level=0.35):
    """Rigid-body drop pool: n^3 grid, water to y < level."""
    return box_3d(n, n, n, 1.0 / n, 2.0, level, 2.0)


def random_boxes(seed, n=128, max_boxes=3, sphere=True):
    """Training scene: 1-3 axis-aligned fluid boxes with extents U[0.2, 0.7]
    and an optional solid sphere obstacle (seeded)."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    lab = _walls((n, n, n))
    x = _centres(n, dx)
    for _ in range(int(rng.integers(1, max_boxes + 1))):
        ext = rng.uniform(0.2, 0.7, 3)
        lo = rng.uniform(0.0, 1.0 - ext)
        hi = lo + ext
        m = ((x >= lo[2]) & (x < hi[2]))[:, None, None] & ((x >= lo[1]) & (x < hi[1]))[None, :, None] & \
            ((x >= lo[0]) & (x < hi[0]))[None, None, :]
        lab[m & (lab != SOLID)] = FLUID
    if sphere and rng.random() < 0.5:
        c = rng.uniform(0.25, 0.75, 3)
        r = rng.uniform(0.06, 0.15)
        zz, yy, xx = np.meshgrid(x, x, x, indexing="ij")
        m = (xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2 < r * r
        lab[m] = SOLID
    return lab


_SM64 = (np.uint64(0x9E3779B97F4A7C15), np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB))


def _splitmix64(x):
    x = x + _SM64[0]
    x = (x ^ (x >> np.uint64(30))) * _SM64[1]
    x = (x ^ (x >> np.uint64(27))) * _SM64[2]
    return x ^ (x >> np.uint64(31))


def _lattice(seed, o, a, b):
    """Lattice value in [0, 1) at integer points (a, b) of octave o."""
    key = (np.uint64(o) << np.uint64(42)) ^ (a.astype(np.uint64) << np.uint64(21)) ^ b.astype(np.uint64)
    return (_splitmix64(np.uint64(seed) ^ _splitmix64(key)) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def value_noise_2d(shape, octaves=4, seed=4):
    """Seeded multi-octave value noise in [0, 1] on an (nz, nx) grid: 4, 8, 16,
    ... lattice cells per octave, smoothstep-weighted bilinear interpolation
    of splitmix64-hashed lattice values, halving amplitudes.  The expressions
    are the ones the GPU scene kernel evaluates (fp_scene_seabed), in the same
    order, so both give the same bits."""
    nz, nx = shape
    kk = np.arange(nz, dtype=np.float64)[:, None]
    ii = np.arange(nx, dtype=np.float64)[None, :]
    out = np.zeros(shape, np.float64)
    amp, tot = 1.0, 0.0
    for o in range(octaves):
        cells = 4 << o
        zs = kk * (float(cells) / float(nz))
        xs = ii * (float(cells) / float(nx))
        z0, x0 = np.broadcast_arrays(zs.astype(np.int64), xs.astype(np.int64))
        fz = zs - zs.astype(np.int64)
        fx = xs - xs.astype(np.int64)
        fz = (fz * fz) * (3.0 - 2.0 * fz)
        fx = (fx * fx) * (3.0 - 2.0 * fx)
        top = _lattice(seed, o, z0, x0) * (1.0 - fx) + _lattice(seed, o, z0, x0 + 1) * fx
        bot = _lattice(seed, o, z0 + 1, x0) * (1.0 - fx) + _lattice(seed, o, z0 + 1, x0 + 1) * fx
        out = out + amp * (top * (1.0 - fz) + bot * fz)
        tot = tot + amp
        amp = amp * 0.5
    return out / tot


def seabed(W=256, H=128, D=256, dx=1.0 / 128, level=0.45, seed=4, bed_base=0.15, bed_amp=0.05, water_xmin=0.0):
    """Large seabed scene: SOLID below bed_base + bed_amp * noise(x, z), water
    to y < level for x >= water_xmin (the wave paddle's side of the tank).
    The parameters are rounded to float32 like fp_scene_seabed's, which
    generates the same labels on the GPU."""
    f = lambda v: float(np.float32(v))
    dx, level, bed_base, bed_amp, water_xmin = f(dx), f(level), f(bed_base), f(bed_amp), f(water_xmin)
    lab = _walls((D, H, W))
    bed = bed_base + bed_amp * value_noise_2d((D, W), 4, seed)  # (D, W) heights
    y = _centres(H, dx)
    x = _centres(W, dx)
    solid = y[None, :, None] < bed[:, None, :]
    water = (y < level)[None, :, None] & (x >= water_xmin)[None, None, :] & ~solid
    lab[solid] = SOLID
    lab[water & (lab != SOLID)] = FLUID
    return lab


def write_labels3d(path, lab):
    """Write a label grid in the reference's 3D file format (reversed order)."""
    D, H, W = lab.shape
    ch = np.array(["S", "F", "A", "S"])[lab]
    with open(path, "w") as f:
        f.write(f"{W} {H} {D}\n")
        for k in range(D - 1, -1, -1):
            for j in range(H - 1, -1, -1):
                f.write(" ".join(ch[k, j, ::-1]) + "\n")


def write_labels2d(path, lab):
    H, W = lab.shape
    ch = np.array(["S", "F", "A", "S"])[lab]
    with open(path, "w") as f:
        f.write(f"{W} {H}\n")
        for j in range(H - 1, -1, -1):
            f.write(" ".join(ch[j]) + "\n")
