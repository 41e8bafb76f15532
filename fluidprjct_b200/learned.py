"""Training and evaluation of the learned pressure preconditioner.

The network (fp_unet_*, csrc/unet.cu and csrc/kernels_unet.cu) is a 3-level 3D
U-Net that maps (cell labels, divergence) to a pressure guess.  Its training
pairs come from the plain PCG solver.  Seeded random fluid boxes (1-3
axis-aligned boxes with extents U[0.2, 0.7], and an optional solid sphere
obstacle) are run as FLIP scenes, and every step contributes (labels, right-hand
side, pressure) to a dataset kept in device memory.  Training runs Adam through
the project's own forward and backward kernels.  torch is used only to hold
device buffers.

Command line (writes the weight file used by FP_SOLVER_PCG_LEARNED):

    python -m fluidprjct_b200.learned --n 128 --scenes 64 --steps-per-scene 64 \\
        --adam-steps 2000 --out fluidprjct_b200/weights/unet3d_128.bin
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import capi
from .scenes import random_boxes

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "unet3d_128.bin")


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the learned preconditioner needs a CUDA device")
    return torch


def generate(n=128, scenes=64, steps_per_scene=64, seed=0, ppc=4, dt=None, tol=1e-7, log=None):
    """(labels uint8, rhs float32, p float32) device tensors of shape
    (scenes * steps_per_scene, n, n, n) from FLIP runs of random_boxes scenes
    solved by the plain FP64 PCG."""
    torch = _torch()
    N = scenes * steps_per_scene
    dev = torch.device("cuda")
    lab = torch.empty((N, n, n, n), dtype=torch.uint8, device=dev)
    rhs = torch.empty((N, n, n, n), dtype=torch.float32, device=dev)
    p = torch.empty((N, n, n, n), dtype=torch.float32, device=dev)
    dx = 1.0 / n
    dt = dt if dt is not None else 0.256 / n  # 0.002 at n = 128: the same CFL number at every n
    k = 0
    t0 = time.time()
    for sc in range(scenes):
        labels = random_boxes(seed * 100003 + sc, n=n)
        s = capi.Solver(dim=3, dx=dx, dt=dt, pic_weight=0.05, solver="pcg", tol=tol, advection="rk2",
                        output_format=capi.OUT_NONE)
        s.set_labels(labels)
        s.seed_particles(ppc, seed * 7919 + sc)
        cells = n ** 3
        for _ in range(steps_per_scene):
            s.step(1)
            s.labels_to_device(lab[k].data_ptr(), cells)
            s.grid_to_device(capi.GRID_RHS, rhs[k].data_ptr(), cells)
            s.grid_to_device(capi.GRID_P, p[k].data_ptr(), cells)
            k += 1
        s.close()
        if log:
            log(f"scene {sc + 1}/{scenes}: {k} pairs, {time.time() - t0:.1f} s")
    return lab, rhs, p


def train(data, adam_steps=2000, lr=5e-4, lr_min=1e-5, seed=0, net=None, log=None, log_every=100):
    """Adam on the relative pressure loss; returns (net, [(step, loss), ...]).
    The learning rate follows a cosine from lr to lr_min."""
    lab, rhs, p = data
    N, D, H, W = lab.shape
    if net is None:
        net = capi.UNet(W, H, D, train=True, seed=seed)
    rng = np.random.default_rng(seed)
    hist = []
    t0 = time.time()
    for it in range(adam_steps):
        k = int(rng.integers(N))
        a = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * it / max(1, adam_steps - 1)))
        want = (it % log_every == 0) or it == adam_steps - 1
        loss = net.train_step(lab[k].data_ptr(), rhs[k].data_ptr(), p[k].data_ptr(), a, want_loss=want)
        if want:
            hist.append((it, loss))
            if log:
                log(f"adam step {it}: loss {loss:.4f} lr {a:.2e} ({time.time() - t0:.1f} s)")
    return net, hist


def eval_loss(net, data, idx):
    """Mean relative loss of the network on the pairs idx (forward only)."""
    lab, rhs, p = data
    out = []
    for k in idx:
        out.append(net.loss_grad(lab[k].data_ptr(), rhs[k].data_ptr(), p[k].data_ptr())[0])
    return float(np.mean(out))


def compare_solvers(labels, rhs, weights, tol=1e-6, dx=None, repeats=3, names=("pcg", "pcg_mg", "pcg_learned")):
    """Solve the same system with the MG-preconditioned PCG from x = 0, with
    the learned initial guess, and with the plain PCG; returns iterations,
    times and residuals of each (device times from fp_step_stats)."""
    D, H, W = labels.shape
    dx = dx if dx is not None else 1.0 / W
    res = {}
    for name in names:
        s = capi.Solver(dim=3, dx=dx, dt=0.002, solver=name, tol=tol, output_format=capi.OUT_NONE)
        s.set_labels(labels)
        if name in ("pcg_learned", "pcg_learned_mixed"):
            s.load_learned(weights)
        times, its = [], []
        for _ in range(repeats):
            _, it, rr, rc = s.pressure_solve(rhs)
            st = s.stats()
            times.append(st["t_pcg"])
            its.append(it)
        res[name] = {"iters": int(its[-1]), "ms": float(np.median(times)), "residual": float(st["residual"]),
                     "fallback": int(st["fallback"]), "learned_ms": float(st["t_learned"]),
                     "guess_relres": float(st["guess_relres"]), "status": int(rc)}
        s.close()
    return res


def time_network(n=128, reps=10):
    """Device time (ms) of one forward pass and one training step of the
    network on an n^3 dam-break-like input, from CUDA events on its stream."""
    torch = _torch()
    net = capi.UNet(n, n, n, train=True, seed=0)
    dev = torch.device("cuda")
    lab = torch.ones((n, n, n), dtype=torch.uint8, device=dev)
    lab[0] = 0
    lab[:, :2] = 0
    lab[:, -max(2, n // 12):] = 2
    gen = torch.Generator(device=dev).manual_seed(0)
    rhs = torch.randn((n, n, n), device=dev, generator=gen) * (lab == 1)
    p = torch.randn((n, n, n), device=dev, generator=gen) * (lab == 1)
    x = torch.zeros_like(rhs)
    torch.cuda.synchronize()
    st = torch.cuda.ExternalStream(net.stream)
    out = {}
    for name, fn in (("forward_ms", lambda: net.forward(lab.data_ptr(), rhs.data_ptr(), x.data_ptr())),
                     ("train_step_ms", lambda: net.train_step(lab.data_ptr(), rhs.data_ptr(), p.data_ptr(), 1e-4))):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    net.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--scenes", type=int, default=64)
    ap.add_argument("--steps-per-scene", type=int, default=64)
    ap.add_argument("--adam-steps", type=int, default=2000)
    ap.add_argument("--lr", type=float, default=5e-4)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--report", default=None, help="JSON summary of the run")
    ap.add_argument("--time", action="store_true", help="only time the network's forward pass and training step")
    ap.add_argument("--reps", type=int, default=10)
    a = ap.parse_args(argv)
    if a.time:
        print(json.dumps({"n": a.n, **time_network(a.n, a.reps)}))
        return
    log = lambda m: print(m, flush=True)
    t0 = time.time()
    data = generate(a.n, a.scenes, a.steps_per_scene, a.seed, log=log)
    t_gen = time.time() - t0
    t1 = time.time()
    net, hist = train(data, a.adam_steps, a.lr, seed=a.seed, log=log)
    t_train = time.time() - t1
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    net.save(a.out)
    held = generate(a.n, 2, 8, a.seed + 1000)
    report = {"pairs": int(data[0].shape[0]), "n": a.n, "adam_steps": a.adam_steps, "gen_s": t_gen,
              "train_s": t_train, "loss_history": hist, "heldout_loss": eval_loss(net, held, range(16))}
    lab = held[0][15].cpu().numpy()
    rhs = held[1][15].cpu().numpy()
    report["heldout_solve"] = compare_solvers(lab, rhs, a.out)
    log(json.dumps(report))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
