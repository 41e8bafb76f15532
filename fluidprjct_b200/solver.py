"""Host-side mirror of the reference's solver class.

``FluidSolver3D`` keeps the interface of Ship-Vano/FluidPrjct's C++ class
(src/FluidSim/FluidSolver3D.cuh:13-186): the constructor
``FluidSolver3D(width, height, depth, dx, dt)``, the public knobs
``PIC_WEIGHT, iterPerFrame, outputFormat, outputTemplate, activeBody,
initialBodyPos, bodyMass``, ``init(labelsPath)`` and ``run(max_steps)``, and
the per-step ``frameStep()``.  Everything runs in the native library through
the C ABI; this class only forwards.
"""
from __future__ import annotations

import os

from . import capi


class FluidSolver3D:
    """Drop-in for ``FluidSolver3D`` (same knobs, same call order)."""

    PARTICLES_PER_CELL = 4  # FluidSolver3D.cuh:71

    def __init__(self, width=5, height=5, depth=5, dx=0.1, dt=0.02, **extra):
        # The constructor's grid size is a placeholder overwritten by init()
        # (main.cpp:21, FluidSolver3D.cu:88), exactly as in the reference.
        self.gridWidth, self.gridHeight, self.gridDepth = width, height, depth
        self.dx, self.dt = dx, dt
        self.PIC_WEIGHT = 0.5       # FluidSolver3D.cuh:156
        self.iterPerFrame = 10      # :157
        self.outputFormat = "PLY"   # :158
        self.outputTemplate = "InputData/particles_"
        self.activeBody = False
        self.initialBodyPos = (0.5, 0.5, 0.5)
        self.bodyMass = 50.0
        self.extra = dict(extra)    # additions: ppc, seed, solver, advection, tol, ...
        self._s = None

    def _config(self):
        fmt = {"PLY": capi.OUT_PLY, "OFF": capi.OUT_OFF, "PLY_BINARY": capi.OUT_PLY_BINARY,
               "NONE": capi.OUT_NONE}.get(self.outputFormat, capi.OUT_OFF)
        kw = dict(dim=3, dx=self.dx, dt=self.dt, pic_weight=self.PIC_WEIGHT, iter_per_frame=self.iterPerFrame,
                  output_format=fmt, output_template=self.outputTemplate, active_body=int(bool(self.activeBody)),
                  body_pos=self.initialBodyPos, body_mass=self.bodyMass, ppc=self.PARTICLES_PER_CELL)
        kw.update(self.extra)
        return capi.default_config(**kw)

    def init(self, labels_path, write_seed_ply=None):
        """init(): read labels, size the grids, seed particles
        (FluidSolver3D.cu:81-204).  The reference writes the seeded set to
        InputData/particles_-1.ply; pass ``write_seed_ply`` to do the same."""
        self._s = capi.Solver(self._config())
        self._s.load_labels(labels_path)
        self.gridWidth, self.gridHeight, self.gridDepth = self._s.dims
        cfg = self._s.cfg
        self._s.seed_particles(cfg.ppc, cfg.seed)
        if write_seed_ply:
            os.makedirs(os.path.dirname(write_seed_ply) or ".", exist_ok=True)
            self._s.save_ply(write_seed_ply, capi.OUT_PLY)

    def run(self, max_steps):
        """run(): max_steps*iterPerFrame + 1 steps with frame output."""
        d = os.path.dirname(self.outputTemplate)
        if d:
            os.makedirs(d, exist_ok=True)
        self._s.run(max_steps)

    def frameStep(self):
        self._s.step(1)

    @property
    def native(self) -> capi.Solver:
        return self._s

    def stats(self):
        return self._s.stats()
