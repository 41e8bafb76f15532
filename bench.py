#!/usr/bin/env python
"""FLIP steps/s on the 128^3 dam break, one B200 per rank.

Workload (the 3D dam break of the benchmark table): 128^3 MAC grid, dx = 1/128,
one-cell SOLID walls, water box x < 0.4, y < 0.6, z < 1 seeded with 8
particles per cell (3,830,400 particles, octant-jittered, seed 1), zero initial
velocity, gravity -9.81, dt = 0.002, FLIP 0.95 (PIC weight 0.05), RK2
advection, 7-point PCG pressure solve (FP32 stencil and vectors, FP64
reductions) to a 1e-6 relative residual.  Synthetic data; the particle state
(2 x 61 MB float4 arrays at 8 ppc) and the grids exceed nothing reusable across steps in
L2 beyond what a real run keeps there, and the particle arrays alone are larger
than the 126 MB L2.

One JSON line on rank 0.  `--impl reference` times the reference's algorithm
on the host cores instead (the CPU oracle port; the reference's own GPU binary
needs cuDSS, which is not installed).  With torchrun (N > 1) each rank runs an
independent replica of the scene on its own GPU (the solver is single-GPU by
design); value = total steps/s, timing = max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FLIP steps/s & PCG time-to-1e-6 at 128³, learned+mixed vs plain on one B200"
N_GRID, DX, DT, PPC, SEED, PIC = 128, 1.0 / 128, 0.002, 8, 1, 0.05


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_GRID)
    ap.add_argument("--ppc", type=int, default=PPC)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--frames", type=int, default=0,
                    help="also time fp_run's frame output (binary and ASCII PLY) over this many frames")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--solver", default="pcg_mg", choices=["pcg", "pcg_mixed", "pcg_mg", "pcg_learned",
                                                           "pcg_learned_mixed"],
                    help="pressure solver of the timed steps")
    ap.add_argument("--no-parity", action="store_true", help="skip the parity leg against the FP64 oracle")
    ap.add_argument("--no-extra", action="store_true", help="skip the 200-step run and the 16 ppc variant")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def max_over_ranks(value, device):
    """The largest of a float over the ranks of the default process group (the
    slowest replica's time); the value itself without a group or with one rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (profiles/), scaled as documented there; None if absent."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"fp_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_scene(n, ppc):
    from fluidprjct_b200 import scenes
    return scenes.dam_break_3d(n)


def new_solver(lab, device, solver="pcg", n=N_GRID, ppc=PPC, warm_start=1):
    from fluidprjct_b200 import capi
    s = capi.Solver(dx=1.0 / n, dt=DT, pic_weight=PIC, advection="rk2", solver=solver, tol=1e-6, max_iters=20000,
                    device=device, output_format=capi.OUT_NONE, warm_start=warm_start)
    s.set_labels(lab)
    if solver in ("pcg_learned", "pcg_learned_mixed"):
        from fluidprjct_b200.learned import DEFAULT_WEIGHTS
        s.load_learned(DEFAULT_WEIGHTS)
    s.seed_particles(ppc, SEED)
    return s


def event_timer(stream_ptr):
    import torch
    st = torch.cuda.ExternalStream(stream_ptr)
    return st, (lambda: torch.cuda.Event(enable_timing=True))


def step_bytes(np_, nc, nf, iters, outer=1):
    """Algorithmic HBM bytes of one whole step (FP32 values, uint8 labels,
    each array read or written once per phase): label 12 Np + 2 Nc, P2G
    24 Np + 24 Nc, RHS 17 Nc, PCG 41 Nf per iteration + 17 Nf per outer
    refinement, projection 29 Nc, G2P + advection 48 Np + 24 Nc; in all
    84 Np + 96 Nc + 41 Nf iters + 17 Nf outer."""
    return 84.0 * np_ + 96.0 * nc + 41.0 * nf * iters + 17.0 * nf * outer


def algorithmic_bytes(np_, nc, nf):
    """Per-phase algorithmic HBM bytes (FP32 values, uint8 labels; each array
    read or written once per phase)."""
    return {
        "label": 16 * np_ * 2 + 8 * np_ + 4 * nc * 3 + 2 * nc,   # read pos/vel, write sorted copies, keys/ranks, counts
        "p2g": 32 * np_ + 24 * (nc * 1.0) + 4 * nc,              # particles in, u,v,w + u*,v*,w* out
        "project": 29 * nc,
        "g2p_advect": 64 * np_ + 24 * nc,                         # pos/vel in+out, u,v,w,u*,v*,w* in
    }


def run_ours(args, rank, local, world):
    import torch
    from fluidprjct_b200 import capi
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    lab = make_scene(args.n, args.ppc)
    s = new_solver(lab, local, args.solver, args.n, args.ppc)
    np_ = s.num_particles
    nc = args.n ** 3
    stream, Ev = event_timer(s.stream)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        s.step(1)
    clocks = Clocks(local)
    barrier()
    clocks.start()
    time.sleep(0.3)
    l0 = s.stats()["kernel_launches"]
    # The K timed steps are one fp_step(K) call, as a caller advances a run:
    # the host issues step k + 1 while the GPU finishes step k (a call per step
    # waits for each step's end and leaves the GPU idle while the host issues
    # the next one, about 47 us per step at 128^3).
    import ctypes as C
    from fluidprjct_b200 import capi
    L = capi.lib()
    e0, e1 = Ev(), Ev()
    e0.record(stream)
    rc = L.fp_step(s._h, args.steps)
    if rc != capi.FP_OK:
        s._check(rc)
    e1.record(stream)
    e1.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    launches = s.stats()["kernel_launches"] - l0
    # Per-step statistics (phase times, iterations, fluid cells) of the same
    # steps, from an identical solver stepped one call per step after the
    # timed region.
    sp = new_solver(lab, local, args.solver, args.n, args.ppc)
    sp.step(args.warmup)
    raw = [capi.FpStepStats() for _ in range(args.steps)]
    for i in range(args.steps):
        rc = L.fp_step(sp._h, 1)
        if rc != capi.FP_OK:
            sp._check(rc)
        L.fp_stats(sp._h, C.byref(raw[i]))
    sp.close()
    per = [r.as_dict() for r in raw]
    ms = max_over_ranks(ms, "cuda")
    ms_step = ms / args.steps
    value = world * args.steps / (ms / 1000.0)

    # ---- roofline of the dominant kernel (the persistent pressure solver) ----
    nf = statistics.mean(p["num_fluid_cells"] for p in per)
    iters = [p["pcg_iters"] for p in per]
    solve_ms = [p["t_pcg"] - p["t_learned"] for p in per]  # the network's share is timed apart
    if args.solver in ("pcg_mg", "pcg_learned"):
        kernel = "k_pcg_mg"
        # per MG-PCG iteration, each array read or written once per pass:
        # Krylov passes 104 B per FLUID cell (w = A z pass: z, r, w; update
        # pass: z, w, p, s, x, r, and the cycle's b and z), level-0 V-cycle
        # 85 B per FLUID cell (seven sweeps of b, x and half of x written;
        # restriction; prolongation), coarser grid-wide levels 5 B per fine
        # cell; the block-solved levels live in shared memory
        solve_bytes = [(189.0 * p["num_fluid_cells"] + 5.0 * nc) * p["pcg_iters"] for p in per]
        note = ("189 B per fluid cell + 5 B per cell per MG-PCG iteration; the kernel is bound by its "
                "~20 grid barriers per iteration and L2 latency (the working set stays in L2), not by HBM")
    else:
        kernel = "k_pcg_cg"
        solve_bytes = [41.0 * p["num_fluid_cells"] * p["pcg_iters"] + 17.0 * p["num_fluid_cells"] * p["outer_iters"]
                       for p in per]
        note = "41 B per fluid cell per iteration + 17 B per fluid cell; working set is L2-resident at 128^3"
    peak, peak_kind = load_peaks()
    solve_gbs = sum(solve_bytes) / (sum(solve_ms) / 1000.0) / 1e9
    traffic = load_traffic()
    phase_ms = {k: statistics.mean(p[k] for p in per) for k in ("t_label", "t_p2g", "t_pressure", "t_project",
                                                                 "t_advect", "t_total")}
    ab = algorithmic_bytes(np_, nc, nf)
    def bw(key, ms):
        g = ab[key] / ms / 1e6
        return {"ms": round(ms, 4), "gbs": round(g, 1), "frac": round(g / peak, 4)}
    phases = {
        "label": bw("label", phase_ms["t_label"]),
        "p2g+save+forces": dict(bw("p2g", phase_ms["t_p2g"]), kernel="k_p2g_accum + k_p2g_finish"),
        "pressure": {"ms": phase_ms["t_pressure"], "solve_ms": statistics.mean(solve_ms),
                     "learned_ms": statistics.mean(p["t_learned"] for p in per), "iters": statistics.mean(iters)},
        "project": dict(bw("project", phase_ms["t_project"]), kernel="k_project"),
        "g2p+advect": dict(bw("g2p_advect", phase_ms["t_advect"]), kernel="k_g2p_advect"),
    }
    sb = statistics.mean(step_bytes(np_, nc, p["num_fluid_cells"], p["pcg_iters"], p["outer_iters"]) for p in per)
    step_gbs = sb / (ms_step / 1000.0) / 1e9
    # DRAM traffic of one captured launch, per iteration of that launch, times
    # the timed solves' mean iterations: the same unit as the algorithmic bytes
    t_launch = (traffic or {}).get(kernel + "_bytes_per_launch")
    t_iters = (traffic or {}).get(kernel + "_iters")
    traffic_launch = (t_launch / t_iters * statistics.mean(iters)) if (t_launch and t_iters) else t_launch
    roofline = {"kernel": kernel + " (persistent cooperative solver)", "bound": "hbm", "achieved": round(solve_gbs, 1),
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(solve_gbs / peak, 4),
                "traffic": round(traffic_launch) if traffic_launch else None,
                "traffic_note": (f"ncu DRAM bytes of one {t_iters}-iteration launch, scaled per iteration to the "
                                 f"timed solves' {statistics.mean(iters):.2f} iterations") if t_iters else None,
                "algorithmic_bytes_per_launch": statistics.mean(solve_bytes), "note": note}
    solver_desc = {
        "pcg": "plain PCG (Jacobi, FP64 vectors)",
        "pcg_mixed": "pcg_mixed (Jacobi PCG, FP32 stencil/vectors, FP64 reductions, FP64 refinement)",
        "pcg_mg": "pcg_mg (flexible PCG with an FP32 multigrid V-cycle preconditioner, FP64 Krylov vectors and "
                  "reductions, warm-started from the previous step's pressure)",
        "pcg_learned": "pcg_learned (flexible PCG: the U-Net as the first preconditioner application, the MG "
                       "V-cycle after it; plain PCG fallback)",
        "pcg_learned_mixed": "pcg_learned_mixed (the U-Net's scaled guess starts pcg_mixed's FP64 refinement; "
                             "plain PCG fallback)",
    }[args.solver]

    out = {"metric": METRIC, "value": round(value, 3), "unit": "steps/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 (FP64 reductions)", "data": "synthetic",
           "config": {"workload": f"3D dam break {args.n}^3, dx=1/{args.n}, fluid x<0.4 y<0.6 z<1, {args.ppc} ppc",
                      "particles": int(np_), "fluid_cells_mean": nf, "dt": DT, "flip": 1 - PIC, "advection": "rk2",
                      "solver": solver_desc,
                      "tol": 1e-6,
                      "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                      "l2": f"inputs larger than L2 (particle arrays 2 x {np_ * 16 / 1e6:.0f} MB + face grids "
                            f"{24 * (args.n + 1) * args.n ** 2 / 1e6:.0f} MB per step)"},
           "ns_per_particle_step": round(ms_step * 1e6 / np_, 3),
           "clocks": clk, "gpu_launches": int(launches), "roofline": roofline, "phases": phases,
           "roofline_step": {"bound": "hbm", "algorithmic_bytes": round(sb), "achieved": round(step_gbs, 1),
                             "peak": peak, "unit": "GB/s", "frac": round(step_gbs / peak, 4),
                             "note": "84 Np + 96 Nc + 41 Nf iters + 17 Nf outer bytes per step over ms_per_step"}}

    # ---- PCG time-to-1e-6 of each solver on the same scene, all from x = 0 (the
    # learned one from its network guess), and MG warm-started as in the step ----
    if not args.no_variants and rank == 0:
        var = {}
        for name, solver, warm in (("pcg", "pcg", 0), ("pcg_mixed", "pcg_mixed", 0), ("pcg_mg", "pcg_mg", 0),
                                   ("pcg_learned", "pcg_learned", 0), ("pcg_learned_mixed", "pcg_learned_mixed", 0),
                                   ("pcg_mg_warm", "pcg_mg", 1)):
            try:
                v = new_solver(lab, local, solver, args.n, args.ppc, warm)
            except Exception as e:  # variant not available in this build
                var[name] = {"unavailable": str(e)}
                continue
            try:
                for _ in range(3):
                    v.step(1)
                st = []
                for _ in range(6):
                    v.step(1)
                    st.append(v.stats())
                var[name] = {"pcg_ms": round(statistics.mean(x["t_pcg"] for x in st), 4),
                             "pressure_ms": round(statistics.mean(x["t_pressure"] for x in st), 4),
                             "iters": statistics.mean(x["pcg_iters"] for x in st),
                             "outer": statistics.mean(x["outer_iters"] for x in st),
                             "residual_max": max(x["residual"] for x in st),
                             "fallback": sum(x["fallback"] for x in st),
                             "learned_ms": round(statistics.mean(x["t_learned"] for x in st), 4),
                             "guess_relres": round(statistics.mean(x["guess_relres"] for x in st), 4)}
            except Exception as e:
                var[name] = {"error": str(e)}
            v.close()
        out["pcg_time_to_1e-6"] = var

    # ---- end to end through the public API with host buffers ----
    if not args.no_e2e:
        pos, vel = s.particles()
        hp = torch.from_numpy(pos).pin_memory()
        hv = torch.from_numpy(vel).pin_memory()
        hpn, hvn = hp.numpy(), hv.numpy()
        k = max(3, min(args.steps, 10))
        barrier()
        a0, a1 = Ev(), Ev()
        a0.record(stream)
        for _ in range(k):
            s.set_particles(hpn, hvn)                      # H2D of the step's input state
            s.step(1)
            s.particles(out=(hpn, hvn))                    # D2H of the step's result, the next input
        a1.record(stream)
        a1.synchronize()
        ems = max_over_ranks(a0.elapsed_time(a1), "cuda")
        out["e2e"] = {"value": round(world * k / (ems / 1000.0), 3), "unit": "steps/s",
                      "h2d_bytes_per_step": int(np_ * 24), "d2h_bytes_per_step": int(np_ * 24), "steps": k,
                      "path": "fp_set_particles(pinned host pos, vel) + fp_step + fp_get_particles"}

    # ---- the configuration's whole run (200 steps from the seeded state) and
    # the 16 ppc variant (7.66 M particles, the configuration's "~8 M") ----
    if not args.no_extra and rank == 0:
        out["run_200_steps"] = timed_run(lab, local, args, 200, 0, args.ppc)
        out["ppc16"] = timed_run(lab, local, args, 20, 5, 16)
        out["other_configs"] = other_configs(local)

    # ---- parity of the timed scene against the FP64 oracle (rank 0, N = 1) ----
    if not args.no_parity and rank == 0 and world == 1:
        out["parity"] = parity_leg(lab, local, args)

    # ---- frame output of fp_run (optional) ----
    if args.frames > 0 and rank == 0:
        out["frame_output"] = frame_output(s, args.frames)

    # ---- CPU baseline (rank 0, N = 1) ----
    if not args.no_cpu and rank == 0 and world == 1:
        out["cpu_baseline"] = cpu_baseline(lab, args.n, args.ppc, args.cpu_seconds)

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    s.close()
    if rank == 0:
        print(json.dumps(out), flush=True)


def timed_run(lab, device, args, steps, warmup, ppc):
    """Device time of `steps` consecutive steps of a fresh solver (after
    `warmup` steps), on the solver's stream."""
    s = new_solver(lab, device, args.solver, args.n, ppc)
    stream, Ev = event_timer(s.stream)
    if warmup:
        s.step(warmup)
    e0, e1 = Ev(), Ev()
    e0.record(stream)
    s.step(steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    st = s.stats()
    n = s.num_particles
    s.close()
    return {"steps": steps, "warmup": warmup, "ppc": ppc, "particles": int(n), "ms": round(ms, 3),
            "steps_per_s": round(steps / (ms / 1000.0), 2), "ns_per_particle_step": round(ms * 1e6 / steps / n, 4),
            "last_step_pcg_iters": st["pcg_iters"], "last_step_residual": st["residual"]}


def _time_steps(s, steps, warmup):
    stream, Ev = event_timer(s.stream)
    s.step(warmup)
    e0, e1 = Ev(), Ev()
    e0.record(stream)
    s.step(steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    st = s.stats()
    return {"steps": steps, "warmup": warmup, "particles": int(s.num_particles), "ms_per_step": round(ms / steps, 4),
            "steps_per_s": round(steps / (ms / 1000.0), 2), "last_pcg_iters": st["pcg_iters"],
            "last_residual": st["residual"], "solve_status": st["solve_status"]}


def other_configs(device):
    """Device-timed steps of the other configurations of the benchmark table
    (each from its seeded state; the warm-up steps are not timed):
    the 2D dam break (64^2, 4 ppc seed 0, dt 0.005, FLIP 0.95, the reference's
    2D step), the rigid-body drop (160^3 pool to y < 0.35, 8 ppc seed 2, sphere
    r 0.12 at half density from (0.5, 0.7, 0.5), SDF collision) and the seabed
    scene (256 x 128 x 256, paddle amplitude 0.05 period 1 s, 8 ppc seed 4,
    dt 0.001)."""
    from fluidprjct_b200 import capi, scenes
    res = {}
    s = capi.Solver(dim=2, dx=1 / 64, dt=0.005, pic_weight=0.05, solver="pcg_mg", tol=1e-6, scheme="ref2d",
                    device=device, output_format=capi.OUT_NONE)
    s.set_labels(scenes.dam_break_2d(64))
    s.seed_particles(4, 0)
    res["dam_break_2d_64"] = _time_steps(s, 100, 0)
    s.close()
    s = capi.Solver(dx=1 / 160, dt=0.002, pic_weight=0.05, solver="pcg_mg", tol=1e-6, body_radius=0.12,
                    body_density=0.5, body_pos=(0.5, 0.7, 0.5), active_body=1, advection="rk2", collision="sdf",
                    device=device, output_format=capi.OUT_NONE)
    s.set_labels(scenes.pool_3d(160, 0.35))
    s.load_sdf(None)
    s.seed_particles(8, 2)
    res["pool_160_sphere"] = _time_steps(s, 20, 3)
    s.close()
    s = capi.Solver(dx=1 / 128, dt=0.001, pic_weight=0.05, solver="pcg_mg", tol=1e-6, advection="rk2", device=device,
                    output_format=capi.OUT_NONE)
    s.scene_seabed(256, 128, 256, level=0.45, bed_base=0.15, bed_amp=0.05, seed=4, water_xmin=0.1)
    s.set_paddle(0.1, 0.05, 1.0)
    s.seed_particles(8, 4)
    res["seabed_256x128x256_paddle"] = _time_steps(s, 20, 3)
    s.close()
    return res


def parity_leg(lab, device, args):
    """The timed configuration against the FP64 oracle (oracle/parity.py):
    step 1 from the seeded state as a whole step (each side its own solver:
    the GPU's MG-PCG to 1e-6, the oracle's FP64 Jacobi PCG to 1e-12), then
    step 2 phase by phase from identical inputs."""
    from oracle import oracle as O
    from oracle import parity
    n = args.n
    s = new_solver(lab, device, args.solver, n, args.ppc)
    o = O.Sim3(n, n, n, 1.0 / n, DT, fp64=True, pic_weight=PIC, tol=1e-12, rk2=True)
    o.set_labels(lab)
    o.set_particles(*s.particles())
    whole = parity.full_step(s, o)
    o.set_particles(*s.particles())
    ph = parity.step_phases(s, o, 1.0 / n)
    s.close()
    o.close()
    r = lambda x: float(f"{x:.3e}")
    return {"labels_bitexact": whole["labels_bitexact"] and ph["labels_bitexact"],
            "u_rel_l2": r(whole["u_rel_l2"]), "v_rel_l2": r(whole["v_rel_l2"]), "w_rel_l2": r(whole["w_rel_l2"]),
            "p_rel_l2": r(whole["p_rel_l2"]), "vel_rel_l2": r(whole["vel_rel_l2"]),
            "pos_rel_l2": r(whole["pos_rel_l2"]),
            "what": "step 1 of the timed scene (GPU MG-PCG to 1e-6) against the oracle's FP64 step (FP64 Jacobi PCG "
                    "to 1e-12); relative L2 over whole arrays",
            "step2_phases": {k: (r(v) if isinstance(v, float) else v) for k, v in ph.items()}}


def frame_output(s, frames):
    """Wall time of fp_run(frames) with one frame per step, for no output,
    binary PLY and ASCII PLY, against the synchronous alternative (the same
    steps, then per frame a download and a file write on the calling
    thread).  fp_run overlaps the writes with the following steps."""
    import copy
    import tempfile

    import numpy as np

    from fluidprjct_b200 import capi
    res = {"frames": frames, "particles": s.num_particles}
    cfg = copy.copy(s.cfg)
    with tempfile.TemporaryDirectory() as tmp:
        for name, fmt, ipf in (("none", capi.OUT_NONE, 1), ("binary", capi.OUT_PLY_BINARY, 1),
                               ("ascii", capi.OUT_PLY, 1), ("binary_every10", capi.OUT_PLY_BINARY, 10),
                               ("ascii_every10", capi.OUT_PLY, 10)):
            cfg.output_format = fmt
            cfg.iter_per_frame = ipf
            cfg.output_template = os.path.join(tmp, name + "_").encode()
            r = capi.Solver(cfg)
            r.set_labels(s.labels())
            pos, vel = s.particles()
            r.set_particles(pos, vel)
            r.step(1)
            t0 = time.perf_counter()
            r.run(frames)  # frames * ipf + 1 steps, frames + 1 files
            res[name + "_ms_per_frame"] = round((time.perf_counter() - t0) * 1000.0 / (frames + 1), 3)
            if fmt != capi.OUT_NONE:
                f0 = os.path.join(tmp, name + "_0.ply")
                res[name + "_bytes_per_frame"] = os.path.getsize(f0)
                # synchronous alternative: the steps, then download and write on this thread
                hp, hv = np.zeros_like(pos), np.zeros_like(vel)
                t0 = time.perf_counter()
                for i in range(frames + 1):
                    r.step(ipf if i else 1)
                    r.particles(out=(hp, hv))
                    capi.lib().fp_write_particle_file(os.path.join(tmp, f"sync_{i}.ply").encode(), capi.ptr(hp),
                                                      capi.ptr(hv), len(hp), fmt)
                res[name + "_sync_ms_per_frame"] = round((time.perf_counter() - t0) * 1000.0 / (frames + 1), 3)
            r.close()
            for f in os.listdir(tmp):
                os.remove(os.path.join(tmp, f))
    return res


def cpu_baseline(lab, n, ppc, seconds):
    """The oracle port of the reference step, all host cores, bounded sample."""
    from oracle import oracle as O
    pos = O.seed3d(lab, 1.0 / n, ppc, SEED)
    sim = O.Sim3(n, n, n, 1.0 / n, DT, fp64=False, pic_weight=PIC, tol=1e-6, rk2=True)
    sim.set_labels(lab)
    sim.set_particles(pos)
    t0 = time.perf_counter()
    steps = 0
    while steps < 1 or (time.perf_counter() - t0 < seconds and steps < 50):
        sim.step(1)
        steps += 1
    el = time.perf_counter() - t0
    return {"value": round(steps / el, 4), "unit": "steps/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"{steps} full steps of the same scene ({len(pos)} particles) from the seeded state, "
                      f"FP32 oracle with FP64 Jacobi-PCG to 1e-6, {el:.1f} s"}


def run_reference(args, rank, world):
    """Reference arm: the reference's algorithm on the host cores (oracle port)."""
    if rank != 0:
        return
    lab = make_scene(args.n, args.ppc)
    from oracle import oracle as O
    pos = O.seed3d(lab, 1.0 / args.n, args.ppc, SEED)
    sim = O.Sim3(args.n, args.n, args.n, 1.0 / args.n, DT, fp64=False, pic_weight=PIC, tol=1e-6, rk2=True)
    sim.set_labels(lab)
    sim.set_particles(pos)
    budget = 150.0
    t_start = time.perf_counter()
    for _ in range(min(args.warmup, 1)):
        sim.step(1)
    t0 = time.perf_counter()
    steps = 0
    while steps < args.steps and (steps < 2 or time.perf_counter() - t_start < budget):
        sim.step(1)
        steps += 1
    el = time.perf_counter() - t0
    v = steps / el
    sample = (f"{steps} of {args.steps} requested steps (time-boxed to {budget:.0f} s) of the same scene, "
              f"{len(pos)} particles, FP32 oracle port with FP64 Jacobi-PCG to 1e-6")
    out = {"metric": METRIC, "value": round(v, 4), "unit": "steps/s", "n_gpus": world, "steps": steps,
           "warmup": min(args.warmup, 1), "ms_per_step": round(1000 * el / steps, 2), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 solve)", "data": "synthetic",
           "impl": "reference",
           "config": {"workload": f"3D dam break {args.n}^3, dx=1/{args.n}, fluid x<0.4 y<0.6 z<1, {args.ppc} ppc",
                      "particles": int(len(pos)), "parallelism": "host cores (OpenMP)"},
           "cpu_baseline": {"value": round(v, 4), "unit": "steps/s", "cores": O.num_threads(), "kind": "port",
                            "sample": sample},
           "e2e": {"value": round(v, 4), "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "note": "the reference's own binary needs cuDSS (absent here); this arm runs the CPU restatement of its step"}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank, local, world = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, local, world)


if __name__ == "__main__":
    main()
