"""fluidprjct_b200 -- B200-native PIC/FLIP liquid solver (sm_100a).

A drop-in for the per-step solve path of Ship-Vano/FluidPrjct: the C ABI in
``include/fluidprjct.h`` (native library ``_lib/libfluidprjct_b200.so``), a
ctypes binding (:mod:`fluidprjct_b200.capi`), a mirror of the reference's
``FluidSolver3D`` class (:mod:`fluidprjct_b200.solver`) and the synthetic
benchmark scenes (:mod:`fluidprjct_b200.scenes`).
"""
from . import capi, scenes  # noqa: F401
from .capi import FluidError, Solver  # noqa: F401
from .solver import FluidSolver3D  # noqa: F401

__all__ = ["capi", "scenes", "Solver", "FluidError", "FluidSolver3D"]
