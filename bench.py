"""Benchmark: fractional time steps of the penalised channel with heat at
256x192x256 (FP64) on B200, plus the FFT Poisson solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  `value` is whole-job time steps per second (the N
ranks run independent replicas: weak scaling), timed with CUDA events on the
solver's stream between barriers, max over ranks.  `e2e` is the same metric
through the public C-ABI with host buffers: pinned-host upload of the job's
inputs, K steps each followed by the device monitor read-back, and the
download of the final state, all inside the timed region.

--impl reference times the CPU restatement of the reference Fortran (the
oracle; the Fortran itself cannot be built here) on all host cores for the
same workload and prints the same line with "impl": "reference".
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "NS steps/s & Poisson GB/s at 256x192x256: FP64 vs mixed, div<=1e-10, 1 B200"
UNIT = "steps/s"
NX, NY, NZ = 256, 192, 256
RE, PR, ETA, WIDTH = 3000.0, 0.71, 1.0e4, 1.5
SPHERE = ((math.pi, 0.0, math.pi / 2), 0.25)
DATA = "synthetic (seeded channel flow + sphere mask; no dataset)"
WORKLOAD = ("sphere256: channel 2pi x 2 x pi, y walls at -1,1 (tanh stretch 2), "
            "256x192x256 cells, sphere R=0.25 at (pi,0,pi/2) by volume penalisation "
            "(eta=1e4, smoothed Heaviside 1.5 dx), heat transfer (sphere T=1, walls T=0), "
            "Re=3000, Pr=0.71, u=1.5(1-y^2)+N(0,0.05^2), CFL 0.5")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dram_traffic():
    """bytes per launch from the committed ncu summary profiles/dram_traffic.txt
    (lines: '<phase> <bytes per launch>'), or {}"""
    out = {}
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.txt")) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and not line.startswith("#"):
                    out[parts[0]] = float(parts[1])
    except OSError:
        pass
    return out


# algorithmic bytes per launch of each phase's kernel (FP64, N interior cells,
# Hs = (nx/2+1)*ny*nz spectral values of 16 B); launches per step in LAUNCHES
def algorithmic_bytes(nx, ny, nz):
    N = nx * ny * nz
    Hs = (nx // 2 + 1) * ny * nz
    return {
        "rhs": 8 * N * 20,        # read u,v,w,T,u_ta x3,4 histories,mask; write u*,v*,w*,T*,4 histories
        "y_vel": 8 * N * 3,       # read rhs + mask, write solution (per field)
        "z_vel": 8 * N * 3,
        "x_vel": 8 * N * 3,
        "y_T": 8 * N * 3,
        "x_T": 8 * N * 3,
        "z_T": 8 * N * 3,
        # read u*,v*,w*, write half spectrum (one unit: the divergence kernel
        # and the x transform it feeds)
        "fft_x_fwd": 8 * N * 3 + 16 * Hs,
        "fft_z_fwd": 2 * 16 * Hs,
        "spn": 2 * 16 * Hs,
        "fft_z_inv": 2 * 16 * Hs,
        "fft_x_inv": 16 * Hs + 8 * N,
        "correct": 8 * N * 18,    # read phi,u*,v*,w*,u_ta x3; write u,v,w,p,ep2 x3,u_ta x3,divu
    }


LINE_PHASES = ("y_vel", "z_vel", "x_vel", "y_T", "x_T", "z_T")
LAUNCHES = {"set_bc": 1, "rhs": 1, "y_vel": 3, "z_vel": 3, "x_vel": 3, "y_T": 1, "x_T": 1,
            "z_T": 1, "set_bc_temp": 1, "fft_x_fwd": 1, "fft_z_fwd": 1, "spn": 1,
            "fft_z_inv": 1, "fft_x_inv": 1, "phibc": 2, "refine": 1, "correct": 1}


class Clocks:
    """nvidia-smi samples (200 ms) while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([s.strip() for s in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def workload_inputs(g, W):
    """Seeded initial fields, CFL time step and the sphere mask of the
    workload on the grid g (numpy only; the GPU arm and the CPU reference arm
    take the same inputs).  The mask is the smoothed Heaviside of
    set_levelset.f:157-170 applied to the exact signed distance of the
    sphere."""
    f = W.channel_state(g, seed=2024, t_bot=0.0, t_top=0.0)
    dt = W.cfl_dt(g, f["u"], f["v"], f["w"])
    c1 = W.smoothed_mask(g, W.sphere_phi0(g, *SPHERE), WIDTH)
    return f, dt, c1


def config_dict(dt):
    """The `config` of the JSON line, identical in both arms."""
    return {"workload": WORKLOAD, "grid": [NX, NY, NZ], "precision": "fp64 plain",
            "mask": "smoothed Heaviside (1.5 dx) of the exact sphere signed distance, "
                    "same array in both arms",
            "initial_state": "seeded noise, then one projection (set_bc + MKP)",
            "l2": "inputs larger than L2 (16 resident FP64 fields of 103 MB)",
            "dt": float("%.12g" % dt)}


def build_case(S, W, torch, precision=0, flags=0, levelset=True):
    """Context with the workload's initial state: the sphere mask, the
    projected field.  With `levelset` the level-set setup (2001 reinitialisation
    sweeps + mask on the GPU, set_levelset.f) is run and timed first; the
    mask the steps use is then replaced by the workload's mask, so that the
    GPU and the CPU reference step from the same array."""
    g = W.grid_arrays(NX, NY, NZ, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    f, dt, c1 = workload_inputs(g, W)
    cfg = S.Config(NX, NY, NZ, dt, RE, PR, ETA, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                   ystretch=2.0, body_force=3.0 / RE, heat_source=0.0, t_bot=0.0, t_top=0.0,
                   t_solid=1.0, precision=precision, flags=flags)
    ctx = S.Context(cfg)
    for k in ("u", "v", "w", "T"):
        ctx.upload(k, f[k])
    ls = None
    if levelset:
        phi0 = W.sphere_phi0(g, *SPHERE)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.levelset(phi0, width=WIDTH, want_phi=False)
        ls = {"seconds": round(time.perf_counter() - t0, 3)}
        ls["mask_max_abs_diff_vs_exact_sdf_mask"] = float(
            np.abs(ctx.download("cellvalue") - c1).max())
    ctx.upload("cellvalue", c1)
    ctx.project()
    ctx.start()
    ctx.sync()
    return g, f, cfg, ctx, ls


# mixed-precision variants reported beside the FP64 line: name -> nse flags
MIXED_VARIANTS = (("mixed", 0),                      # default: FP64 Poisson solve
                  ("mixed_fp64_lines", 64),          # + NSE_FLAG_LINES64
                  ("mixed_fp32_poisson", 512))       # NSE_FLAG_POISSON32: FP32 FFTs + 1
                                                     # FP64 refinement pass


def run_mixed(S, W, torch, stream, args, fp64_ms):
    """Speed of each mixed variant (same timing as the FP64 line) and its
    accuracy against an FP64 run of the same seed after args.acc_steps steps:
    relative L2 of u, v, w, T, of the joint velocity, and the largest
    post-projection divergence seen after any of those steps (also split into
    the first step, where the penalisation stops the flow inside the sphere
    impulsively and the pressure is largest, and the rest), with the same
    figures for the FP64 run."""
    out = {}
    ref = None

    def divs(c, n):
        d = []
        for _ in range(n):
            c.step(1)
            d.append(c.monitor()["max_divu"])
        return d

    if args.acc_steps > 0:
        _, _, _, ref, _ = build_case(S, W, torch, levelset=False)
        rd = divs(ref, args.acc_steps)
        refs = {k: ref.download(k) for k in ("u", "v", "w", "T")}
        ref.close()
        out["fp64_reference"] = {"accuracy_steps": args.acc_steps, "max_divu": max(rd),
                                 "max_divu_step1": rd[0],
                                 "max_divu_after_step1": max(rd[1:] or [0.0])}
    for name, flags in MIXED_VARIANTS:
        _, _, _, ctx, _ = build_case(S, W, torch, precision=S.MIXED, flags=flags,
                                        levelset=False)
        ctx.set_stream(stream.cuda_stream)
        with torch.cuda.stream(stream):
            ctx.step(args.warmup)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        # per-phase times from as many further steps with the phase events on
        # (the events themselves cost a few microseconds each, so they stay
        # out of the timed steps)
        ctx.profile(args.steps)
        ctx.step(args.steps)
        torch.cuda.synchronize()
        phases, nprof = ctx.phase_times()
        ctx.close()
        rec = {"steps_per_s": round(args.steps / (ms / 1e3), 3),
               "ms_per_step": round(ms / args.steps, 4),
               "speedup_vs_fp64": round(fp64_ms / ms, 3),
               "phases_ms_per_step": {k: round(v / max(1, nprof), 4) for k, v in phases.items()}}
        if args.acc_steps > 0:
            _, _, _, ctx, _ = build_case(S, W, torch, precision=S.MIXED, flags=flags,
                                        levelset=False)
            md = divs(ctx, args.acc_steps)
            got = {k: ctx.download(k) for k in ("u", "v", "w", "T")}
            ctx.close()
            rel = {k: float(np.linalg.norm(got[k] - refs[k]) / np.linalg.norm(refs[k]))
                   for k in got}
            num = sum(np.linalg.norm(got[k] - refs[k]) ** 2 for k in ("u", "v", "w"))
            den = sum(np.linalg.norm(refs[k]) ** 2 for k in ("u", "v", "w"))
            rec.update({"accuracy_steps": args.acc_steps, "max_divu": max(md),
                        "max_divu_step1": md[0], "max_divu_after_step1": max(md[1:] or [0.0]),
                        "rel_l2_vs_fp64": rel,
                        "velocity_rel_l2_vs_fp64": float(math.sqrt(num / den))})
        out[name] = rec
    return out


def run_big(S, W, torch, stream, args):
    """The 512x256x512 mixed-precision workload: the sphere geometry of the
    main workload on the finer grid, the mixed form (default: FP64 Poisson
    solve) and the FP64 form stepped args.big_steps penalised steps from the
    same projected seeded field and the same mask; per-step divergence of
    both, relative L2 of u, v, w, T and of the joint velocity of the mixed run
    against the FP64 run, and the speed of both.  Then the seeded N(0,1)
    right-hand side (dy-weighted mean removed) solved by the FP64 Poisson
    solve, with the relative residual of the discrete operator it inverts."""
    nx, ny, nz = 512, 256, 512
    g = W.grid_arrays(nx, ny, nz, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    f = W.channel_state(g, seed=512, t_bot=0.0, t_top=0.0)
    dt = W.cfl_dt(g, f["u"], f["v"], f["w"])
    c1 = W.smoothed_mask(g, W.sphere_phi0(g, *SPHERE), WIDTH)
    res = {"grid": [nx, ny, nz], "steps": args.big_steps, "dt": dt,
           "mask": "smoothed Heaviside (1.5 dx) of the exact sphere signed distance"}
    out = {}
    for name, prec in (("fp64", S.FP64), ("mixed", S.MIXED)):
        cfg = S.Config(nx, ny, nz, dt, RE, PR, ETA, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                       ystretch=2.0, body_force=3.0 / RE, heat_source=0.0, t_bot=0.0,
                       t_top=0.0, t_solid=1.0, precision=prec)
        with S.Context(cfg) as ctx:
            ctx.set_stream(stream.cuda_stream)
            for k in ("u", "v", "w", "T"):
                ctx.upload(k, f[k])
            ctx.upload("cellvalue", c1)
            ctx.project()
            ctx.start()
            divs = []
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            ms = 0.0
            for _ in range(args.big_steps):
                e0.record(stream)
                ctx.step(1)
                e1.record(stream)
                d = ctx.monitor()
                ms += e0.elapsed_time(e1)
                divs.append(d["max_divu"])
            out[name] = {k: ctx.download(k) for k in ("u", "v", "w", "T")}
            res[name] = {"ms_per_step": round(ms / max(1, args.big_steps), 4),
                         "max_divu": max(divs), "max_divu_step1": divs[0] if divs else None}
            if prec == S.FP64:
                rhs = W.poisson_rhs(g, seed=513)
                ctx.upload("phi", rhs)
                ctx.poisson()
                phi = ctx.download("phi")
                res["poisson_rhs"] = {"seed": 513, "solve": "fp64",
                                      "relative_residual": poisson_residual(g, phi, rhs)}
    a, b = out["mixed"], out["fp64"]
    res["mixed"]["rel_l2_vs_fp64"] = {k: float(np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k]))
                                      for k in a}
    num = sum(np.linalg.norm(a[k] - b[k]) ** 2 for k in ("u", "v", "w"))
    den = sum(np.linalg.norm(b[k]) ** 2 for k in ("u", "v", "w"))
    res["mixed"]["velocity_rel_l2_vs_fp64"] = float(math.sqrt(num / den))
    res["mixed"]["speedup_vs_fp64"] = round(res["fp64"]["ms_per_step"] /
                                            res["mixed"]["ms_per_step"], 3)
    return res


def poisson_residual(g, phi, rhs):
    """||L phi - rhs|| / ||rhs|| on the interior, L the 7-point operator the
    spectral solve inverts (periodic second differences in x and z, the
    stretched-grid second difference in y with PHIBC's Neumann ghosts); the
    plane mean of the residual at J = NY, the mean-mode row that SP0B's
    marching does not enforce, is left out."""
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    P = phi
    i, j, k = slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1)
    dx, dy, dz = g["dx"], g["dy"], g["dz"]
    dx12, dy12, dz12 = g["dx12"], g["dy12"], g["dz12"]
    L = ((P[2:nx + 2, j, k] - P[i, j, k]) / dx12[1:nx + 1, None, None] -
         (P[i, j, k] - P[0:nx, j, k]) / dx12[0:nx, None, None]) / dx[1:nx + 1, None, None]
    L += ((P[i, 2:ny + 2, k] - P[i, j, k]) / dy12[None, 1:ny + 1, None] -
          (P[i, j, k] - P[i, 0:ny, k]) / dy12[None, 0:ny, None]) / dy[None, 1:ny + 1, None]
    L += ((P[i, j, 2:nz + 2] - P[i, j, k]) / dz12[None, None, 1:nz + 1] -
          (P[i, j, k] - P[i, j, 0:nz]) / dz12[None, None, 0:nz]) / dz[None, None, 1:nz + 1]
    r = L - rhs[i, j, k]
    r[:, ny - 1, :] -= r[:, ny - 1, :].mean()
    return float(np.linalg.norm(r) / np.linalg.norm(rhs[i, j, k]))


def replica_rate(ms_local, steps, world, device="cpu"):
    """Whole-job rate of `world` replicas that each timed `steps` steps in
    ms_local: the slowest rank's time (all-reduce MAX over the process group;
    one value per rank, gloo on CPU or nccl on the GPU) and world*steps
    divided by it.  Returns (ms_max, steps_per_s)."""
    ms_max = float(ms_local)
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([ms_max], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    return ms_max, world * steps / (ms_max / 1e3)


def shard_cases(n, rank, world):
    """Indices of the ensemble cases of this rank: the n cases are dealt
    round-robin over the world ranks (whole cases per GPU, no exchange while
    they run)."""
    return list(range(rank, n, world))


def gather_case_scalars(local, n, width, world, device="cpu"):
    """Per-case scalars of the whole ensemble in case order.  `local` maps
    this rank's case indices to `width` floats; every case belongs to exactly
    one rank, so one all-reduce (SUM) of an n x width tensor in which each
    rank fills its own rows gathers them (gloo on CPU, nccl on the GPU)."""
    import torch
    t = torch.zeros((n, width), dtype=torch.float64)
    for i, vals in local.items():
        t[i] = torch.tensor(vals, dtype=torch.float64)
    if world > 1:
        import torch.distributed as dist
        t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [tuple(float(x) for x in row) for row in t.cpu()]


def run_ensemble(S, W, torch, stream, args, rank=0, world=1, device="cpu"):
    """Batched ensemble: args.ens_cases cases drawn by seed (grids among
    64^3..160x128x160, 1-3 spheres or cubes, Re_bulk in [1000, 5000], own
    noise), in FP64 and in the mixed form with the FP64 Poisson solve and FP64
    line arithmetic.  Aggregate case-steps/s of args.steps steps replayed from
    the captured graph on 8 streams, beside the same cases stepped one after
    the other on one stream; per-case error of the mixed form against FP64
    after args.acc_steps steps.  With world > 1 the cases are sharded over the
    ranks (shard_cases), the aggregate rate uses the slowest rank's time and
    the per-case scalars are gathered (gather_case_scalars)."""
    import torch.distributed as dist
    mine = shard_cases(args.ens_cases, rank, world)
    cases = [W.ensemble_case(7000 + i) for i in mine]

    def slowest(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def build(prec, flags):
        out = []
        for g, f, phi0, Re, _ in cases:
            dt = W.cfl_dt(g, f["u"], f["v"], f["w"])
            cfg = S.Config(g["nx"], g["ny"], g["nz"], dt, Re, PR, ETA, 2 * math.pi, 2.0, math.pi,
                           y0=-1.0, ystretch=2.0, body_force=3.0 / Re, heat_source=0.0,
                           t_bot=1.0, t_top=0.0, t_solid=1.0, precision=prec, flags=flags)
            c = S.Context(cfg)
            for k in ("u", "v", "w", "T"):
                c.upload(k, f[k])
            c.levelset(phi0, width=WIDTH, want_phi=False)
            c.project()
            c.start()
            out.append(c)
        return out

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return slowest(e0.elapsed_time(e1))

    shapes = gather_case_scalars({i: (g["nx"], g["ny"], g["nz"]) for i, (g, *_) in zip(mine, cases)},
                                 args.ens_cases, 3, world, device)
    cells = int(sum(a * b * c for a, b, c in shapes))
    res = {"cases": args.ens_cases, "cells": cells, "streams": args.ens_streams,
           "grids": sorted({tuple(int(x) for x in sh) for sh in shapes})}
    if world > 1:
        res["ranks"] = world
        res["sharding"] = ("whole cases dealt round-robin over the ranks; aggregate rate over "
                           "the slowest rank's time; per-case scalars gathered by one all-reduce")
    finals = {}
    divs = {}
    for name, prec, flags in (("fp64", S.FP64, 0), ("mixed", S.MIXED, 64)):
        ctxs = build(prec, flags)
        for c in ctxs:
            c.set_stream(stream.cuda_stream)
            c.step(1)  # Euler start and the mask tables, outside the timing
        seq_ms = timed(lambda: [c.step(args.steps) for c in ctxs])
        if ctxs:
            with S.Ensemble(ctxs, nstreams=args.ens_streams) as ens:
                ens.set_stream(stream.cuda_stream)
                ens.step(2)
                ens.sync()
                ms = timed(lambda: ens.step(args.steps))
                ens.sync()
                if args.acc_steps > 0:
                    ens.step(args.acc_steps - 1 - args.steps - 2)
                    ens.sync()
        else:
            ms = timed(lambda: None)
        finals[name] = [{k: c.download(k) for k in ("u", "v", "w", "T")} for c in ctxs]
        divs[name] = {i: (c.monitor()["max_divu"],) for i, c in zip(mine, ctxs)}
        for c in ctxs:
            c.close()
        div_all = gather_case_scalars(divs[name], args.ens_cases, 1, world, device)
        res[name] = {"case_steps_per_s": round(args.ens_cases * args.steps / (ms / 1e3), 1),
                     "cell_steps_per_s": round(cells * args.steps / (ms / 1e3), 1),
                     "sequential_case_steps_per_s":
                         round(args.ens_cases * args.steps / (seq_ms / 1e3), 1),
                     "graph_speedup_vs_sequential": round(seq_ms / ms, 3),
                     "max_divu_at_end": max(d[0] for d in div_all)}
    errs = {}
    for i, a, b in zip(mine, finals["mixed"], finals["fp64"]):
        num = sum(np.linalg.norm(a[k] - b[k]) ** 2 for k in ("u", "v", "w"))
        den = sum(np.linalg.norm(b[k]) ** 2 for k in ("u", "v", "w"))
        errs[i] = (math.sqrt(num / den),
                   float(np.linalg.norm(a["T"] - b["T"]) / np.linalg.norm(b["T"])))
    allerr = gather_case_scalars(errs, args.ens_cases, 2, world, device)
    vel = [e[0] for e in allerr]
    tem = [e[1] for e in allerr]
    # steps behind the comparison: 1 + steps (sequential) + 2 + steps + the rest
    res["mixed_vs_fp64_after_steps"] = 3 + 2 * args.steps + max(0, args.acc_steps - 3 - args.steps)
    res["mixed_velocity_rel_l2"] = {"max": max(vel), "median": float(np.median(vel))}
    res["mixed_T_rel_l2"] = {"max": max(tem), "median": float(np.median(tem))}
    return res


def run_dft_gemm(S, W, torch, stream, n=64, reps=50):
    """The tensor-core question for small transforms (the smallest ensemble grid,
    n^3 with n = 64): one Poisson solve of the library (its own radix FFTs in
    x and z, SPN, inverse) against the four transform passes of a solve done
    as dense DFT matrix products through cuBLAS (torch.matmul): the x passes
    as a real (n^2 x n) by (n x 2(n/2+1)) product, the z passes as a complex
    (n x n) by (n x (n/2+1) n) product, each twice (forward and inverse), in
    FP64 (the form's precision) and in TF32 (the tensor-core precision the
    FP32 form would use).  CUDA events on one stream, after warm-up."""
    g = W.grid_arrays(n, n, n, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    cfg = S.Config(n, n, n, 1.0, 1.0, 1.0, 0.0, 2 * math.pi, 2.0, math.pi, y0=-1.0, ystretch=2.0)
    dev = torch.device("cuda")

    def timed(fn):
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    with S.Context(cfg) as ctx:
        ctx.set_stream(stream.cuda_stream)
        ctx.upload("phi", W.poisson_rhs(g, 3))
        ours = timed(ctx.poisson)
    h = n // 2 + 1
    out = {"n": n, "reps": reps, "library_solve_ms": round(ours, 5)}
    for name, dt in (("fp64", torch.float64), ("tf32", torch.float32)):
        torch.backends.cuda.matmul.allow_tf32 = name == "tf32"
        with torch.cuda.stream(stream):
            xr = torch.randn(n * n, n, dtype=dt, device=dev)
            fr = torch.randn(n, 2 * h, dtype=dt, device=dev)
            zc = torch.randn(2 * n, h * n, dtype=dt, device=dev)
            fz = torch.randn(2 * n, 2 * n, dtype=dt, device=dev)

        def passes():
            torch.matmul(xr, fr)   # x pass (real samples -> half spectrum)
            torch.matmul(fz, zc)   # z pass (complex as a 2n x 2n real block)

        t = 2 * timed(passes)
        out[f"gemm_{name}_ms"] = round(t, 5)
        out[f"gemm_{name}_flop"] = 2 * (2 * n * n * n * 2 * h + 2 * (2 * n) ** 2 * h * n)
    torch.backends.cuda.matmul.allow_tf32 = False
    out["note"] = ("GEMM times cover the four transform passes only (no SPN, no sample "
                   "packing); the library time is a whole solve")
    return out


def run_adjoint(S, W, torch, stream, args):
    """Discrete adjoint at args.adj_grid^3: the sphere of the main workload at
    the same physical size, walls at T = 1 (y = -1) and T = 0 (y = 1), sphere
    T = 1; args.adj_steps FP64 steps from the projected noisy channel,
    checkpointed every 20 steps in device memory; J = mean wall heat flux at
    y = -1 over the last 100 steps.  dJ/dc1 from one adjoint sweep, checked
    along args.adj_dirs seeded N(0,1) directions against central finite
    differences of J with step 1e-6."""
    n = args.adj_grid
    g = W.grid_arrays(n, n, n, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    f = W.channel_state(g, seed=2025, t_bot=1.0, t_top=0.0)
    dt = W.cfl_dt(g, f["u"], f["v"], f["w"])
    cfg = S.Config(n, n, n, dt, RE, PR, ETA, 2 * math.pi, 2.0, math.pi, y0=-1.0, ystretch=2.0,
                   body_force=3.0 / RE, heat_source=0.0, t_bot=1.0, t_top=0.0, t_solid=1.0)
    N = args.adj_steps
    avg_from = max(1, N - 99)
    res = {"grid": [n, n, n], "steps": N, "checkpoint_every": 20, "avg_from": avg_from,
           "objective": "mean over the last 100 steps of the area-weighted wall heat flux at "
                        "y = -1, thc (T(i,1,k) - T(i,0,k)) / dy12(0)",
           "walls": "T = 1 at y = -1, T = 0 at y = 1, sphere T = 1", "dt": dt}
    with S.Context(cfg) as ctx:
        ctx.set_stream(stream.cuda_stream)
        for k in ("u", "v", "w", "T"):
            ctx.upload(k, f[k])
        ctx.levelset(W.sphere_phi0(g, *SPHERE), width=WIDTH, want_phi=False)
        ctx.project()
        ctx.start()
        c1 = ctx.download("cellvalue")
        names = ("u", "v", "w", "T", "u_ta", "v_ta", "w_ta", "u_pre", "v_pre", "w_pre", "T_pre")
        st0 = {k: ctx.download(k) for k in names}
        l0 = ctx.step_index

        def reset(c):
            for k in names:
                ctx.upload(k, st0[k])
            ctx.upload("cellvalue", c)
            ctx.step_index = l0

        with S.Adjoint(ctx, N, checkpoint_every=20, avg_from=avg_from) as adj:
            # one untimed forward run first (first-use costs: kernel loading,
            # the context's side streams), then the timed one
            reset(c1)
            adj.objective()
            reset(c1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            J0 = adj.objective()
            t_fwd = time.perf_counter() - t0
            reset(c1)
            t0 = time.perf_counter()
            J, grad = adj.gradient()
            t_grad = time.perf_counter() - t0
            rng = np.random.default_rng(4242)
            eps = 1e-6

            def central(d, e):
                reset(c1 + e * d)
                Jp = adj.objective()
                reset(c1 - e * d)
                return (Jp - adj.objective()) / (2 * e)

            # central differences at eps, and Richardson's combination of eps
            # and eps/2, (4 D(eps/2) - D(eps)) / 3, which cancels the eps^2
            # truncation term (the response to a perturbation of every cell
            # of the mask is strongly nonlinear: the plain error scales as eps^2)
            errs, errs_c, rows = [], [], []
            t0 = time.perf_counter()
            for _ in range(args.adj_dirs):
                d = rng.standard_normal(c1.shape)
                f1 = central(d, eps)
                f2 = central(d, eps / 2)
                fr = (4.0 * f2 - f1) / 3.0
                ad = float(np.sum(grad * d))
                errs.append(abs(fr - ad) / abs(fr))
                errs_c.append(abs(f1 - ad) / abs(f1))
                rows.append([fr, f1, ad])
            t_fd = time.perf_counter() - t0
    res.update({"J": J, "J_forward_only": J0, "forward_s": round(t_fwd, 3),
                "gradient_s": round(t_grad, 3),
                "gradient_over_forward": round(t_grad / t_fwd, 2),
                "fd_directions": args.adj_dirs, "fd_step": eps,
                "fd_rel_err": {"max": max(errs), "median": float(np.median(errs)),
                               "kind": "Richardson-extrapolated central differences "
                                       "(steps 1e-6 and 5e-7)"},
                "central_fd_rel_err": {"max": max(errs_c), "median": float(np.median(errs_c)),
                                       "kind": "central differences, step 1e-6"},
                "fd_richardson_central_adjoint_first": rows[:4], "fd_s": round(t_fd, 2),
                "grad_l2": float(np.linalg.norm(grad))})
    return res


def summary(line):
    """The headline figures of the line in a few keys (printed last, so a
    truncated log tail still shows them)."""
    out = {"fp64_steps_per_s": line["value"], "e2e_steps_per_s": line["e2e"]["value"],
           "poisson_ms": line["poisson"]["ms_per_solve"],
           "poisson_frac_of_hbm": line["poisson"]["frac_of_hbm"]}
    mp = line.get("mixed_precision") or {}
    for name, rec in mp.items():
        if name == "fp64_reference":
            continue
        out[name] = {"speedup_vs_fp64": rec.get("speedup_vs_fp64"),
                     "max_divu": rec.get("max_divu"),
                     "velocity_rel_l2_vs_fp64": rec.get("velocity_rel_l2_vs_fp64")}
    big = line.get("mixed_512x256x512")
    if big:
        out["mixed_512"] = {"speedup_vs_fp64": big["mixed"]["speedup_vs_fp64"],
                            "max_divu": big["mixed"]["max_divu"],
                            "velocity_rel_l2_vs_fp64": big["mixed"]["velocity_rel_l2_vs_fp64"]}
    if line.get("parity"):
        out["parity_max_rel_l2"] = line["parity"]["max_rel_l2"]
        out["parity_pass"] = line["parity"]["pass"]
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from vtkmakecompare_b200 import solver as S
    from vtkmakecompare_b200 import workload as W

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    g, f0, cfg, ctx, ls = build_case(S, W, torch)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---------------------------------------------------- device-resident steps
    with torch.cuda.stream(stream):
        ctx.step(args.warmup)
    torch.cuda.synchronize()
    barrier()
    n0 = S.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local_rank) as clk:
        torch.cuda.synchronize()
        barrier()
        e0.record(stream)
        ctx.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
    launches = S.launch_count() - n0
    ms = e0.elapsed_time(e1)
    ms_max, steps_s = replica_rate(ms, args.steps, world, dev)
    mon = ctx.monitor()
    # per-phase times (roofline, phases_ms_per_step) from K further steps with
    # the phase events on, outside the timed region
    ctx.profile(args.steps)
    with torch.cuda.stream(stream):
        ctx.step(args.steps)
    torch.cuda.synchronize()
    phases, nprof = ctx.phase_times()

    # ---------------------------------------------------------- Poisson solve
    ctx.upload("phi", W.poisson_rhs(g, 7))
    with torch.cuda.stream(stream):
        ctx.poisson()
    torch.cuda.synchronize()
    npois = max(5, args.steps)
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    barrier()
    p0.record(stream)
    for _ in range(npois):
        ctx.poisson()
    p1.record(stream)
    torch.cuda.synchronize()
    pms = max_over_ranks(p0.elapsed_time(p1)) / npois
    Hs = (NX // 2 + 1) * NY * NZ
    BP = 2 * 8 * NX * NY * NZ + 4 * 16 * Hs
    # the opt-in solves on the same right-hand side (one GPU only): the SPN
    # through TMA tiles and the three-pass solve
    pvar = {}
    if world == 1:
        for name, flag in (("spn_tma", S.FLAG_SPN_TMA), ("three_pass", S.FLAG_POISSON3)):
            vcfg = S.Config(NX, NY, NZ, 1.0, 1.0, 1.0, 0.0, 2 * math.pi, 2.0, math.pi, y0=-1.0,
                            ystretch=2.0, flags=flag)
            with S.Context(vcfg) as vc:
                vc.set_stream(stream.cuda_stream)
                vc.upload("phi", W.poisson_rhs(g, 7))
                vc.poisson()
                torch.cuda.synchronize()
                p0.record(stream)
                for _ in range(npois):
                    vc.poisson()
                p1.record(stream)
                torch.cuda.synchronize()
                vms = p0.elapsed_time(p1) / npois
                vc.sync()
            pvar[name] = {"ms_per_solve": round(vms, 4),
                          "frac_of_hbm": round(BP / (vms / 1e3) / 1e9 / peaks()[0], 4)}

    # ------------------------------------------------------------------ e2e
    # the job through the public API from pinned host buffers: upload the
    # inputs (u, v, w, T, mask), K steps each followed by the monitor
    # read-back, download of the final state (u, v, w, p, T)
    shape = (NX + 2, NY + 2, NZ + 2)
    pin = {k: torch.from_numpy(np.ascontiguousarray(f0[k].ravel(order="F"))).pin_memory()
           for k in ("u", "v", "w", "T")}
    c1 = ctx.download("cellvalue")
    pin["cellvalue"] = torch.from_numpy(np.ascontiguousarray(c1.ravel(order="F"))).pin_memory()
    outs = {k: torch.empty(int(np.prod(shape)), dtype=torch.float64).pin_memory()
            for k in ("u", "v", "w", "p", "T")}
    h2d = sum(t.numel() * 8 for t in pin.values())
    d2h = sum(t.numel() * 8 for t in outs.values()) + 48 * args.steps
    mon_ok = True

    def job():
        nonlocal mon_ok
        for k, t in pin.items():
            ctx.upload_ptr(k, t.data_ptr())
        ctx.step_index = 1
        ctx.start()
        for _ in range(args.steps):
            ctx.step(1)
            m = ctx.monitor()
            mon_ok = mon_ok and m["nonfinite"] == 0
        for k, t in outs.items():
            ctx.download_ptr(k, t.data_ptr())

    job()  # warm
    torch.cuda.synchronize()
    barrier()
    q0 = torch.cuda.Event(enable_timing=True)
    q1 = torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    job()
    q1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(q0.elapsed_time(q1))
    barrier()

    # ------------------------------------------------- mixed-precision form
    mixed = None
    if not args.no_mixed:
        mixed = run_mixed(S, W, torch, stream, args, ms)

    # ------------------------------------------------------- batched ensemble
    ensemble = None
    if args.ens_cases > 0:
        ensemble = run_ensemble(S, W, torch, stream, args, rank, world, dev)

    dft_gemm = None
    if args.dft_gemm and rank == 0:
        dft_gemm = run_dft_gemm(S, W, torch, stream)

    # ---------------------------------------- 512x256x512 mixed-precision leg
    big = None
    if args.big_steps > 0 and rank == 0:
        big = run_big(S, W, torch, stream, args)

    # ------------------------------------------------------ discrete adjoint
    adjoint = None
    if args.adj_steps > 0:
        adjoint = run_adjoint(S, W, torch, stream, args)

    # ---------------------------------- parity against the CPU oracle + CPU baseline
    parity, cpu = None, None
    if rank == 0 and args.parity_steps > 0:
        parity, cpu = run_parity(S, W, torch, args.parity_steps)

    if rank != 0:
        ctx.close()
        return None

    # ------------------------------------------------------------- roofline
    algo = algorithmic_bytes(NX, NY, NZ)
    peak, peak_kind = peaks()
    per_launch = {k: phases[k] / max(1, nprof) / LAUNCHES[k] for k in phases}
    # the fast form runs the four components' line chains on concurrent
    # streams and reports the whole block (12 line passes) under y_vel: not
    # one kernel, so it is left out of the dominant-kernel choice
    concurrent_lines = all(phases[k] <= 0.05 * phases["y_vel"] for k in LINE_PHASES[1:])
    dominant = max((k for k in phases
                    if k in algo and not (concurrent_lines and k in LINE_PHASES)),
                   key=lambda k: phases[k])
    t_launch_s = per_launch[dominant] / 1e3
    achieved = algo[dominant] / t_launch_s / 1e9
    traffic = dram_traffic().get(dominant)
    poisson = {"solves_per_s": round(world * 1e3 / pms, 2), "ms_per_solve": round(pms, 4),
               "algorithmic_bytes": BP, "gbs": round(BP / (pms / 1e3) / 1e9, 1),
               "frac_of_hbm": round(BP / (pms / 1e3) / 1e9 / peak, 4)}
    if pvar:
        poisson["opt_in_solves"] = pvar
    line = {
        "metric": METRIC,
        "value": round(steps_s, 3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_max / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": DATA,
        "config": config_dict(cfg.dt),
        "parallelism": f"replicas x{world}",
        "gpu_launches": int(launches),
        "levelset_setup": ls,
        "ensemble": ensemble,
        "adjoint": adjoint,
        "phases_ms_per_step": {k: round(v / max(1, nprof), 4) for k, v in phases.items()},
        "phases_note": ("the line passes of u, v, w and T run as four concurrent chains; "
                        "y_vel holds the whole line block" if concurrent_lines else
                        "from K further steps with the phase events on, which run every "
                        "pass on one stream in order; the timed steps run the four line "
                        "chains concurrently"),
        "mixed_precision": mixed,
        "mixed_512x256x512": big,
        "dft_as_gemm_64": dft_gemm,
        "max_divu": mon["max_divu"],
        "poisson": poisson,
        "parity": parity,
        "e2e": {"value": round(world * args.steps / (e2e_ms / 1e3), 3), "unit": UNIT,
                "h2d_bytes_per_step": int(h2d / args.steps),
                "d2h_bytes_per_step": int(d2h / args.steps),
                "note": "job of K steps: pinned H2D of u,v,w,T,mask + K x (step + monitor "
                        "read-back) + D2H of u,v,w,p,T"},
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1),
                     "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": algo[dominant],
                     "ms_per_launch": round(per_launch[dominant], 4)},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }
    line["summary"] = summary(line)
    ctx.close()
    return line


class _OGrid:
    """grid dict -> the attribute object the oracle binding expects"""

    def __init__(self, g):
        self.__dict__.update(g)


def oracle_case(O, g, f, dt, c1):
    """The CPU restatement of the reference time loop on the workload's
    inputs: same fields, mask and dt, the initial projection (set_bc + MKP),
    the AB2 history copy (nse_dominik.f:246-257)."""
    s = O.Solver(g, dt, RE, PR, ETA, force=3.0 / RE, source=0.0, tbot=0.0, ttop=0.0,
                 tsolid=1.0)
    for k in ("u", "v", "w", "T"):
        s.f[k][...] = f[k]
    s.cellvalue[..., 0] = c1
    s.project()
    s.start()
    return s


PARITY_FIELDS = ("u", "v", "w", "p", "T", "u_ta", "v_ta", "w_ta", "u_pre", "v_pre", "w_pre",
                 "T_pre")


def run_parity(S, W, torch, nsteps):
    """The GPU FP64 step (default fast form, a fresh context) against the CPU
    oracle on identical inputs: both project the same seeded field with the
    same mask, take one warm step and then `nsteps` timed steps.  Relative L2
    of every state field after 1 + nsteps steps (bound 1e-10) and the largest
    post-projection divergence of both.  The oracle's timed steps (faithful
    mode: the reference's per-line dense matrix zeroing, all host threads)
    are the CPU baseline."""
    from oracle import oracle as O
    g, f, cfg, ctx, _ = build_case(S, W, torch, levelset=False)
    c1 = ctx.download("cellvalue")
    ctx.step(1 + nsteps)
    mon = ctx.monitor()
    got = {k: ctx.download(k) for k in PARITY_FIELDS}
    gdiv = np.abs(ctx.download("divu")).max()
    ctx.close()
    O.set_faithful(True)
    s = oracle_case(O, _OGrid(g), f, cfg.dt, c1)
    s.step(1)  # warm (first touch of the work arrays) and the Euler start
    t0 = time.perf_counter()
    s.step(nsteps)
    el = time.perf_counter() - t0
    rel = {k: float(np.linalg.norm(got[k] - s.f[k]) / np.linalg.norm(s.f[k]))
           for k in PARITY_FIELDS}
    odiv = float(np.abs(s.f["divu"]).max())
    umax = float(np.abs(s.f["u"]).max())
    dx = float(g["dx"][1])
    parity = {"steps": 1 + nsteps, "grid": [NX, NY, NZ], "form": "fp64 fast (default)",
              "rel_l2_vs_oracle": rel, "max_rel_l2": max(rel.values()), "bound": 1e-10,
              "max_divu_gpu": float(mon["max_divu"]), "max_abs_divu_field_gpu": float(gdiv),
              "max_divu_oracle": odiv, "divu_bound": 1e-12 * max(1.0, umax / dx),
              "pass": bool(max(rel.values()) <= 1e-10 and
                           mon["max_divu"] <= 1e-12 * max(1.0, umax / dx))}
    cpu = {"value": round(nsteps / el, 4), "unit": UNIT, "cores": O.num_threads(),
           "kind": "port",
           "sample": f"{nsteps} full FP64 time steps of the 256x192x256 workload ({el:.1f} s) "
                     "after the projection and one warm step; oracle faithful mode, the same "
                     "run the parity block compares against"}
    return parity, cpu


def run_reference(args, rank, world):
    """The CPU reference arm: the oracle (C++/OpenMP restatement of the
    reference Fortran, faithful mode) on all host threads, on the same
    inputs as the GPU arm (grid from the oracle's own SET_C restatement,
    the same seeded fields, dt and mask), each step a full time step."""
    if rank != 0:
        return None
    from oracle import oracle as O
    from vtkmakecompare_b200 import workload as W  # numpy input generators only
    og = O.Grid(NX, NY, NZ, 2 * math.pi, 2.0, math.pi, y0=-1.0, gamma=2.0)
    g = {k: getattr(og, k) for k in ("x", "x12", "y", "y12", "z", "z12", "dx", "dx12", "dy",
                                     "dy12", "dz", "dz12")}
    g.update(nx=NX, ny=NY, nz=NZ, xl=og.xl, yl=og.yl, zl=og.zl)
    f, dt, c1 = workload_inputs(g, W)
    O.set_faithful(True)
    s = oracle_case(O, og, f, dt, c1)
    s.step(max(1, args.warmup))
    t0 = time.perf_counter()
    s.step(args.steps)
    el = time.perf_counter() - t0
    v = args.steps / el
    return {
        "metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * el / args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": DATA,
        "config": config_dict(dt),
        "impl": "reference",
        "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": O.num_threads(),
                         "kind": "port",
                         "sample": f"{args.steps} full time steps after {max(1, args.warmup)} "
                                   "warm steps; C++/OpenMP restatement of the reference "
                                   "(the Fortran + FFTW build is not available here)"},
        "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--parity-steps", type=int, default=10,
                    help="timed steps of the GPU-vs-oracle parity run at the bench size "
                         "(its oracle timing is the CPU baseline; 0 skips both)")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--ens-cases", type=int, default=32,
                    help="cases of the batched-ensemble measurement (0 skips it)")
    ap.add_argument("--ens-streams", type=int, default=8,
                    help="streams the batched ensemble's cases are spread over")
    ap.add_argument("--adj-steps", type=int, default=400,
                    help="forward steps of the adjoint measurement (0 skips it)")
    ap.add_argument("--adj-grid", type=int, default=128)
    ap.add_argument("--dft-gemm", action="store_true",
                    help="also time 64-point transforms as dense DFT GEMMs (cuBLAS) "
                         "against the library's own transform")
    ap.add_argument("--adj-dirs", type=int, default=16)
    ap.add_argument("--big-steps", type=int, default=100,
                    help="steps of the 512x256x512 FP64-vs-mixed leg (0 skips it)")
    ap.add_argument("--acc-steps", type=int, default=100,
                    help="steps of the mixed-vs-FP64 accuracy comparison")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        line = run_ours(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
