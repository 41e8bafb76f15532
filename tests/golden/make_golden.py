"""Generate the golden fixtures of tests/golden/ from the reference checkout.

Run once where the reference is available:
    python tests/golden/make_golden.py /path/to/FluidPrjct
It writes, from the reference's own data and test files:
  particles_m1.npz      InputData/particles_-1.ply positions (44,144 x 3, float32)
  labels_fixtures.npz   the label grids of InputData/labels_*.txt (uint8) and
                        their cell counts
  labels_simple3d.txt   InputData/labels_simple3d.txt (30 bytes, reader input)
  labels_simple.txt     InputData/labels_simple.txt (27 bytes, reader input)
  kat_cudss_5x5.json    the 5x5 SPD known-answer system of src/FluidSim/test.cu
                        (:261-290 matrix and rhs, :378-383 expected x = 1..5)
The label parser used here is independent of both the oracle and the product.
"""
from __future__ import annotations

import json
import os
import re
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_labels(path):
    # Header integers, then one label per non-blank character (the reference
    # reads `file >> char`, which skips whitespace).
    text = open(path).read()
    toks = text.split()
    if len(toks) >= 3 and toks[2].isdigit():
        W, H, D = map(int, toks[:3])
        ch = "".join(toks[3:])[:W * H * D]
        lab = np.zeros((D, H, W), np.uint8)
        code = {"S": 0, "F": 1, "A": 2}
        t = 0
        for k in range(D - 1, -1, -1):          # FluidSolver3D.cu:139-141
            for j in range(H - 1, -1, -1):
                for i in range(W - 1, -1, -1):
                    lab[k, j, i] = code[ch[t]]
                    t += 1
        return lab
    W, H = map(int, toks[:2])
    ch = "".join(toks[2:])[:W * H]
    lab = np.zeros((H, W), np.uint8)
    code = {"S": 0, "F": 1, "A": 2}
    t = 0
    for j in range(H - 1, -1, -1):              # FluidSolver2D.cu:71-96
        for i in range(W):
            lab[j, i] = code[ch[t]]
            t += 1
    return lab


def main(ref):
    inp = os.path.join(ref, "InputData")
    # particles_-1.ply (ascii, x y z)
    lines = open(os.path.join(inp, "particles_-1.ply")).read().split("\n")
    end = lines.index("end_header")
    pos = np.array([[float(t) for t in l.split()] for l in lines[end + 1:] if l.strip()], np.float32)
    np.savez_compressed(os.path.join(HERE, "particles_m1.npz"), pos=pos)

    arrays, counts = {}, {}
    for name in ["labels_simple3d.txt", "labels_simple.txt", "labels_colimn.txt", "labels_3d_sphere.txt",
                 "labels_bathymetry.txt"]:
        lab = parse_labels(os.path.join(inp, name))
        key = name[:-4]
        arrays[key] = lab
        counts[key] = {"shape": list(lab.shape), "F": int((lab == 1).sum()), "S": int((lab == 0).sum()),
                       "A": int((lab == 2).sum())}
    np.savez_compressed(os.path.join(HERE, "labels_fixtures.npz"), **arrays)
    for small in ["labels_simple3d.txt", "labels_simple.txt"]:
        shutil.copyfile(os.path.join(inp, small), os.path.join(HERE, small))

    src = open(os.path.join(ref, "src", "FluidSim", "test.cu")).read()
    def grab(name):
        return [float(x) for x in re.findall(name + r"\[i\+\+\]\s*=\s*([-0-9.]+)", src)]
    kat = {
        "source": "src/FluidSim/test.cu:261-290,378-383",
        "offsets": [int(x) for x in grab("csr_offsets_h")],
        "cols": [int(x) for x in grab("csr_columns_h")],
        "vals": grab("csr_values_h"),
        "b": grab("b_values_h"),
        "x": [1.0, 2.0, 3.0, 4.0, 5.0],
        "tol": 2e-15,
    }
    assert len(kat["offsets"]) == 6 and len(kat["cols"]) == 8 and len(kat["vals"]) == 8 and len(kat["b"]) == 5
    meta = {"particles_m1": {"n": int(len(pos)), "dx": 0.02, "cells": 11036, "per_cell": 4,
                             "source": "InputData/particles_-1.ply, InputData/config.json:3 (dx)"},
            "labels": counts, "kat": kat}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FLUIDPRJCT_REFERENCE", "")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout>  (or set FLUIDPRJCT_REFERENCE)")
    main(root)
