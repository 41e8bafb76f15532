"""Build the native library ``fluidprjct_b200/_lib/libfluidprjct_b200.so`` and
the ``FluidGPU`` driver executable beside it (``_lib/FluidGPU``, the reference's
``main.cpp`` over the C ABI, linked to the library with an ``$ORIGIN`` rpath).

Every CUDA source is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) with IEEE division and square
root (no fast-math), so cell keys match the reference bit for bit.  The
library is built in-tree so that it travels with the repository.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libfluidprjct_b200.so")
DRIVER = os.path.join(LIBDIR, "FluidGPU")
BUILD = os.path.join(HERE, "_build")

SOURCES = [
    "kernels_sort.cu",
    "kernels_p2g.cu",
    "kernels_pressure.cu",
    "kernels_advect.cu",
    "kernels_body.cu",
    "kernels_mg.cu",
    "kernels_unet.cu",
    "kernels_unet_tma.cu",
    "kernels_ref2d.cu",
    "kernels_scene.cu",
    "kernels_extrap.cu",
    "unet.cu",
    "solver.cu",
    "noalloc.cu",
    "io.cpp",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "fluidprjct.h"))
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc, "-ccbin", _host_cxx(), *ARCH, *NVCC_FLAGS, "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc, "-ccbin", _host_cxx(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-ldl",
               "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    main = os.path.join(CSRC, "fluidgpu_main.cpp")
    header = os.path.join(HERE, "..", "include", "fluidprjct.h")
    if force or _stale(DRIVER, [main, header, LIB]):
        cmd = [_host_cxx(), "-O2", "-std=c++17", "-Wall", main, "-o", DRIVER, "-L" + LIBDIR, "-lfluidprjct_b200",
               "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
