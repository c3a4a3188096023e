#!/usr/bin/env python
"""Benchmark of the collision + transport time step on B200.

Workload (the metric's configuration): spatially inhomogeneous periodic run,
64 x-cells on [0,1) per GPU, N = 32 velocity grid on [-6,6)^2 (L = 6,
R = 3.75), J = 16 angles, M = 16 Gauss-Legendre radial nodes, h = 1/64,
dt = 0.4 h / L (CFL 0.4), Bext = 0, FP64, seeded Gaussian-mixture initial
state.  One step = one Strang step (1/2 transport, midpoint collision on
every cell, 1/2 transport) = 2 cell-collision evaluations per cell.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (launched by torchrun) every rank owns 64 cells of a 64N-cell
periodic domain (weak scaling) and exchanges 2-cell halos with its ring
neighbours over NCCL before each half step of transport.

value  : cell-collision evals/s, whole job, state resident in HBM, device-timed
         (CUDA events per step, L2 flushed before each step, max over ranks)
e2e    : same metric through the upstream C API (InhomStepPeriodic on host
         buffers, H2D + D2H inside every step) at N = 1; through the sharded
         step with host staging at N > 1
--impl reference : the upstream C sources (compiled here with the project's
         CPU FFTW-API shim) on the host cores, bounded sample per step.

Extra blocks of the JSON line at N = 1: `precision_form` (the FP32 form on
the same workload, with its error against FP64) and `config2_sample` (64 of
the 1024 x-cells of the N = 64, J = M = 32 precision-form configuration, FP64
and FP32 timed alike; --no-config2 skips it), `config3_sample` (256 homogeneous
instances of mixed N, RK4, FP64 and FP32; --no-config3 skips it), and `surrogate` (a Fourier
neural operator trained here on homogeneous relaxation data, used for the
collision half of the same Strang steps with the exact operator as judge
every 10th step and as per-cell fallback; --no-surrogate skips it);
--surrogate-n64 adds the same at N = 64, J = M = 32 (`surrogate_n64`).
"""
import argparse
import importlib.util
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "inhom-quantum-boltzmann-fourier-c_b200")
METRIC = "cell-collision evals/s & sim steps/s vs plain FP64 GPU at <=1e-5 rel err"
UNIT = "cell-collision evals/s"


def _import(name, path):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(args):
    return dict(N=args.grid, J=args.J, M=args.M, L=6.0, R=3.75, cells=args.cells,
                h=1.0 / args.cells, dt=0.4 * (1.0 / args.cells) / 6.0, seed=1)


def config_json(wl, world, flush):
    return {"workload": f"inhomogeneous periodic Strang step, {wl['cells']} x-cells per GPU, N={wl['N']} "
                        f"(padded {2 * wl['N']}), J={wl['J']} angles, M={wl['M']} Gauss-Legendre nodes, "
                        f"L={wl['L']}, R={wl['R']}, h=1/{wl['cells']}, dt=0.4h/L, midpoint collision, FP64",
            "cells_per_gpu": wl["cells"], "cells_total": wl["cells"] * world, "N": wl["N"], "J": wl["J"], "M": wl["M"],
            "parallelism": f"x-cells sharded over {world} GPU(s), 2-cell halo exchange" if world > 1 else "1 GPU",
            "l2": flush}


# ---------------------------------------------------------------------------
# CPU baseline: the upstream C code (oracle/_ref) on the host cores

def _ref_eval_worker(args):
    """one cell-collision evaluation (CcInt + CdInt) of the upstream code"""
    J, M, L, R, Wv = args
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import orc
    r = orc.Ref(J, M, L, R)
    WF = orc.ref_to_fourier(Wv)
    t = time.perf_counter()
    r.cc(WF)
    r.cd(WF)
    return time.perf_counter() - t


def cpu_sample(wl, procs, seed_offset=0):
    """bounded sample: `procs` processes each evaluate C[W] of one cell"""
    qbgpu = _import("qbgpu", os.path.join(PKG, "qbgpu.py"))
    W = qbgpu.gaussian_mixture_state(wl["N"], wl["L"], seed=wl["seed"], ncells=wl["cells"])
    jobs = [(wl["J"], wl["M"], wl["L"], wl["R"], W[(i + seed_offset) % wl["cells"]]) for i in range(procs)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        pool.map(_ref_eval_worker, jobs)
    wall = time.perf_counter() - t0
    return procs / wall, wall


def ref_kind():
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import orc
    return "reference" if orc.ref_available() else None


# ---------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.p = None
        self.path = os.path.join("/tmp", f"qb_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.fh.close()

    def summary(self):
        if self.p is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------

def i3_flops_per_term(N):
    """algorithmic FP64 flops of the I3 kernel per (cell, quadrature term):
    4 padded spectra (0.75 of a full 2N x 2N FFT each: half the rows are zero)
    + 16 (i, j) pairs x (IFFT2 + FFT2) at 5 n log2 n per transform, plus the
    pointwise products (19 flops per padded point per pair, 6 per N-point
    per source)."""
    P = 2 * N
    F = 5.0 * P * P * math.log2(P * P)
    return 4 * 0.75 * F + 32 * F + 16 * 19 * P * P + 4 * 6 * N * N


def captured_traffic(kernel, wl):
    """DRAM bytes (read + write) per launch of `kernel` on this workload from
    the committed ncu capture (profiles/dram_traffic.json, written from
    dram__bytes_read.sum + dram__bytes_write.sum of one launch), or None"""
    path = os.path.join(REPO, "profiles", "dram_traffic.json")
    try:
        rows = json.load(open(path))
    except (OSError, ValueError):
        return None
    for r in rows:
        if r.get("kernel") == kernel and all(r.get(k) == wl[k] for k in ("N", "J", "M", "cells")):
            return r["bytes_per_launch"]
    return None


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    qbgpu = _import("qbgpu", os.path.join(PKG, "qbgpu.py"))
    qd = _import("qb_dist", os.path.join(PKG, "qb_dist.py"))
    L = qbgpu.lib()
    wl = workload(args)
    N, cells = wl["N"], wl["cells"]

    Wall = qbgpu.gaussian_mixture_state(N, wl["L"], seed=wl["seed"], ncells=cells * world)
    W0 = torch.from_numpy(Wall[rank * cells:(rank + 1) * cells].copy()).cuda()
    q, ws = qbgpu.Quad(N, wl["J"], wl["M"], wl["L"], wl["R"]), qbgpu.Workspace(N)
    B = torch.zeros((cells, 3), dtype=torch.float64, device="cuda")
    bufs = [W0.clone(), torch.empty_like(W0)]

    if world == 1:
        def step(Win, Wout):
            qbgpu.inhom_step(ws, q, Win, wl["h"], wl["dt"], B, out=Wout)
    else:
        sharded = qd.ShardedStrang(cells, (4, N, N), torch.float64, W0.device,
                                   lambda ext, out: qbgpu.transport(ext, wl["L"], wl["h"], 0.5 * wl["dt"], out=out),
                                   lambda c, i: qbgpu.fourier_collision(ws, q, c, wl["dt"], B[i:i + c.shape[0]]))

        def step(Win, Wout):
            sharded.step(Win, out=Wout)

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")     # 256 MB > 126 MB L2
    for i in range(args.warmup):
        step(bufs[i % 2], bufs[(i + 1) % 2])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    launches0 = L.qb_launch_count()
    replays0 = ws.graph_replays
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    cur = args.warmup % 2
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record()
            step(bufs[cur], bufs[1 - cur])
            evs[k][1].record()
            cur = 1 - cur
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    launches = L.qb_launch_count() - launches0
    replays = ws.graph_replays - replays0
    ms = sum(a.elapsed_time(b) for a, b in evs)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * cells * 2 * args.steps / (ms * 1e-3)
    steps_per_s = args.steps / (ms * 1e-3)

    # per-kernel device times: a second pass over the same steps with kernel
    # profiling on (CUDA events around every launch; steps then launch kernel
    # by kernel instead of replaying their graph)
    L.qb_profile_reset()
    L.qb_profile_enable(1)
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()
        step(bufs[cur], bufs[1 - cur])
        cur = 1 - cur
    torch.cuda.synchronize()
    L.qb_profile_enable(0)

    # dominant kernel: the I3 cluster kernel
    import ctypes
    kms, kn = ctypes.c_double(), ctypes.c_long()
    L.qb_profile_read(b"i3_cluster", ctypes.byref(kms), ctypes.byref(kn))
    tot_ms, tot_n = ctypes.c_double(), ctypes.c_long()
    L.qb_profile_read(b"", ctypes.byref(tot_ms), ctypes.byref(tot_n))
    L.qb_fp64_peak_tflops.restype = ctypes.c_double
    peak = L.qb_fp64_peak_tflops()
    per_launch_ms = kms.value / max(1, kn.value)
    flops_launch = cells * wl["J"] * wl["M"] * i3_flops_per_term(N)
    achieved = flops_launch / (per_launch_ms * 1e-3) / 1e12
    i3name = "k_i3p" if N == 32 else ("k_i3_128" if N == 64 else "k_i3")
    i3desc = {"k_i3p": "k_i3p (I3 quadrature sums, 2-CTA cluster, accumulators in tensor memory)",
              "k_i3_128": "k_i3_128 (I3 quadrature sums, grids split over CTA pairs)",
              "k_i3": "k_i3 (I3 quadrature sums, 4-CTA cluster)"}[i3name]
    roofline = {"bound": "fp64", "kernel": i3desc, "achieved": round(achieved, 3),
                "peak": round(peak, 3), "unit": "TFLOP/s", "frac": round(achieved / peak, 4) if peak > 0 else None,
                "peak_source": "measured live: DFMA loop on every SM (qb_fp64_peak_tflops); MEASURED_PEAKS.json has no FP64 figure",
                "flops_per_launch": flops_launch, "launch_ms": round(per_launch_ms, 4), "launches": kn.value,
                "launch_timing": "CUDA events around each launch, in a second pass over the same steps launched kernel by kernel "
                                 "(the timed steps replay CUDA graphs)",
                "share_of_step": round(kms.value / max(1e-9, tot_ms.value), 4),
                "traffic": captured_traffic(i3name, wl)}
    state_bytes = cells * 4 * N * N * 8
    hbm = {"bound": "hbm", "note": "whole step: transport reads+writes the state twice, collision reads W^ and writes C (FP64)",
           "bytes_per_step": 4 * state_bytes + 2 * cells * 3 * 4 * N * N * 16,
           "achieved": round((4 * state_bytes + 2 * cells * 3 * 4 * N * N * 16) * steps_per_s / 1e9, 3), "unit": "GB/s"}

    # end to end through the public API with host buffers
    e2e = run_e2e(args, wl, qbgpu, qd, world, rank, q, ws, B, Wall)
    prec = None
    if world == 1 and not args.no_precision_form:
        prec = run_precision_form(args, wl, qbgpu, q, B, Wall, flush, value)
    big = None
    if world == 1 and not args.no_config2:
        big = run_config2_sample(args, qbgpu, flush, cells=args.config2_cells)
    big3 = None
    if world == 1 and not args.no_config3:
        big3 = run_config3_sample(args, qbgpu, flush, ninst=args.config3_ninst)
    dmm = None
    if world == 1 and not args.no_dftmma:
        dmm = run_dftmma_sample(args, qbgpu, flush)
    sur = None
    if world == 1 and not args.no_surrogate:
        sur = run_surrogate(args, wl, qbgpu, q, B, Wall, flush, value)
    sur64 = None
    if world == 1 and args.surrogate_n64:
        sur64 = run_surrogate64(args, qbgpu, flush)

    line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian mixture)",
            "config": config_json(wl, world, "flushed: 256 MB written before every timed step"),
            "sim_steps_per_s": round(steps_per_s, 4), "roofline": roofline, "hbm_view": hbm, "e2e": e2e,
            "gpu_launches": launches, "graph_replays": replays, "clocks": clk.summary()}
    if prec is not None:
        line["precision_form"] = prec
    if big is not None:
        line["config2_sample"] = big
    if big3 is not None:
        line["config3_sample"] = big3
    if dmm is not None:
        line["dftmma_sample"] = dmm
    if sur is not None:
        line["surrogate"] = sur
    if sur64 is not None:
        line["surrogate_n64"] = sur64
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        kind = ref_kind()
        procs = max(1, min(os.cpu_count() or 1, args.cpu_procs))
        if kind is not None:
            rate, wall = cpu_sample(wl, procs)
            line["cpu_baseline"] = {"value": round(rate, 5), "unit": UNIT, "cores": procs, "kind": kind,
                                    "sample": f"{procs} processes x 1 cell-collision evaluation (CcInt + CdInt) of the upstream C code, "
                                              f"{wall:.1f} s wall; FFTs through the project's CPU FFTW-API shim (FFTW absent)"}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_config2_sample(args, qbgpu, flush, cells=64, steps=2, warmup=1):
    """A bounded sample of the precision-form configuration: N = 64 (padded
    128 x 128), J = M = 32, seeded Gaussian mixture, periodic Strang steps on
    `cells` of its 1024 x-cells (h, dt as for 1024 cells), FP64 and the FP32
    form timed alike (CUDA events, L2 flushed before every step), with the
    FP32 form's error against FP64 on the collision operator of the sample and
    how many cell evaluations of its timed steps ran the I3 sums in real form."""
    import torch
    N, J, M, L, R = 64, 32, 32, 6.0, 3.75
    h = 1.0 / 1024
    dt = 0.4 * h / L
    q = qbgpu.Quad(N, J, M, L, R)
    W0 = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=2, ncells=cells)).cuda()
    B = torch.zeros((cells, 3), dtype=torch.float64, device="cuda")
    out = {"workload": f"N={N} (padded {2 * N}), J={J}, M={M}, L={L}, R={R}, {cells} of the 1024 x-cells, h=1/1024, "
                       f"dt=0.4h/L, periodic Strang step; {steps} timed steps after {warmup} warm-up per precision",
           "unit": UNIT}
    for prec in (64, 32):
        ws = qbgpu.Workspace(N, precision=prec)
        bufs = [W0.clone(), torch.empty_like(W0)]
        for i in range(warmup):
            qbgpu.inhom_step(ws, q, bufs[i % 2], h, dt, B, out=bufs[(i + 1) % 2])
        torch.cuda.synchronize()
        ws.i3_forms(reset=True)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        cur = warmup % 2
        for k in range(steps):
            flush.zero_()
            evs[k][0].record()
            qbgpu.inhom_step(ws, q, bufs[cur], h, dt, B, out=bufs[1 - cur])
            evs[k][1].record()
            cur = 1 - cur
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs) / steps
        out[f"f{prec}"] = {"value": round(cells * 2 / (ms * 1e-3), 3), "ms_per_step": round(ms, 3),
                           "sim_steps_per_s_at_1024_cells": round(1e3 / (ms * 1024 / cells), 5)}
        if prec == 32:
            real, total = ws.i3_forms()      # cell evaluations of the timed steps, by I3 form
            out["f32"]["i3_real_form_cells"] = f"{real} of {total}"
        del ws
    out["speedup_f32_vs_f64"] = round(out["f32"]["value"] / out["f64"]["value"], 4)
    Wf = torch.empty((cells, 4, N, N), dtype=torch.complex128, device="cuda")
    qbgpu._check(qbgpu.lib().qb_to_fourier(N, 4 * cells, qbgpu._ptr(W0), qbgpu._ptr(Wf), qbgpu._stream()), "qb_to_fourier")
    ws64, ws32 = qbgpu.Workspace(N), qbgpu.Workspace(N, precision=32)
    cc64, cd64 = qbgpu.collision_operators(ws64, q, Wf)
    cc32, cd32 = qbgpu.collision_operators(ws32, q, Wf)

    def rel(a, b):
        a, b = a.cpu().numpy().ravel(), b.cpu().numpy().ravel()
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out["rel_err_f32_vs_f64"] = {"Cc_l2": rel(cc32, cc64), "Cd_l2": rel(cd32, cd64)}
    if args.config2_long_steps > 0:
        out["long_run"] = config2_long_run(qbgpu, q, W0, h, dt, args.config2_long_cells, args.config2_long_steps)
    return out


def config2_long_run(qbgpu, q, W0, h, dt, cells, steps):
    """The FP32 form against FP64 after `steps` Strang steps on the first
    `cells` x-cells of the sample (a periodic line of those cells, h and dt of
    the 1024-cell domain): relative error of W and of Cc, Cd on the final FP64
    state; and, with the conservation correction on, the relative drift of the
    total mass, momentum and energy of the FP32 run."""
    import torch
    N = q.N
    L = 6.0
    Ws = W0[:cells].contiguous()
    B = torch.zeros((cells, 3), dtype=torch.float64, device="cuda")
    runs = {}
    for name, prec, cons in (("f64", 64, False), ("f32", 32, False), ("f32_conserving", 32, True)):
        ws = qbgpu.Workspace(N, precision=prec, conserve=cons)
        a, b = Ws.clone(), torch.empty_like(Ws)
        for _ in range(steps):
            qbgpu.inhom_step(ws, q, a, h, dt, B, out=b)
            a, b = b, a
        torch.cuda.synchronize()
        runs[name] = a

    def rel(x, y, o):
        x, y = x.cpu().numpy().ravel(), y.cpu().numpy().ravel()
        return float(np.linalg.norm(x - y, o) / np.linalg.norm(y, o))

    def totals(W):
        d = qbgpu.diagnostics(W, L).cpu().numpy()       # the library's moment kernel (FP64)
        mass = d[:, 0]
        mom = mass[:, None] * d[:, 4:6]
        energy = mass * (d[:, 6] + 0.5 * (d[:, 4] ** 2 + d[:, 5] ** 2))
        return mass.sum(), mom.sum(axis=0), energy.sum()
    m0, p0, e0 = totals(Ws)
    m1, p1, e1 = totals(runs["f32_conserving"])
    Wf = qbgpu.to_fourier(runs["f64"])
    ws64, ws32 = qbgpu.Workspace(N), qbgpu.Workspace(N, precision=32)
    cc64, cd64 = qbgpu.collision_operators(ws64, q, Wf)
    cc32, cd32 = qbgpu.collision_operators(ws32, q, Wf)
    return {"what": f"{steps} Strang steps of the first {cells} x-cells (a periodic line of them, h = 1/1024), FP32 form against FP64",
            "W_rel_l1": rel(runs["f32"], runs["f64"], 1), "W_rel_l2": rel(runs["f32"], runs["f64"], 2),
            "Cc_rel_l2_on_final_state": rel(cc32, cc64, 2), "Cd_rel_l2_on_final_state": rel(cd32, cd64, 2),
            "conserving_f32_drift": {"mass": abs(m1 - m0) / abs(m0),
                                     "momentum": float(np.linalg.norm(p1 - p0) / max(np.linalg.norm(p0), abs(m0))),
                                     "energy": abs(e1 - e0) / abs(e0)},
            "bounds": {"C": 1e-5, "drift": 1e-9}}


def run_config3_sample(args, qbgpu, flush, ninst=256, steps=2, warmup=1):
    """A sample of the mixed-size batch configuration: `ninst` independent
    homogeneous instances with N drawn from the configuration's sizes (16, 24,
    32, 48, 64, 96, 128 with weights 0.1, 0.1, 0.25, 0.2, 0.2, 0.1, 0.05;
    N = 24, 48, 96, 128 run on the any-N engine), seeded Gaussian mixtures, RK4
    steps of dt = 0.01 (J = M = 16), FP64 and the FP32 form timed alike (CUDA
    events, L2 flushed before every step), with the FP32 form's deviation from
    FP64 on the final states; then all `config3_big` instances in the FP32
    form."""
    import torch
    L, R, J, M, dt = 6.0, 3.75, 16, 16, 0.01
    rng = np.random.default_rng(3)
    sizes_all = [16, 24, 32, 48, 64, 96, 128]
    w = np.array([0.1, 0.1, 0.25, 0.2, 0.2, 0.1, 0.05])
    if args.config3_sizes:                 # a subset of the sizes (profiling), weights renormalised
        keep = [int(x) for x in args.config3_sizes.split(",")]
        w = np.array([wi for n, wi in zip(sizes_all, w) if n in keep])
        sizes_all = [n for n in sizes_all if n in keep]
    sizes = rng.choice(sizes_all, size=ninst, p=w / w.sum())
    Wf = [qbgpu.to_fourier(torch.from_numpy(qbgpu.gaussian_mixture_state(int(n), L, seed=3000 + i, ncells=1)).cuda())[0].contiguous()
          for i, n in enumerate(sizes)]
    out = {"workload": f"{ninst} homogeneous instances, N in (16, 24, 32, 48, 64, 96, 128) with weights "
                       f"(0.1, 0.1, 0.25, 0.2, 0.2, 0.1, 0.05), J={J}, M={M}, RK4 dt={dt}, {steps} timed steps after {warmup} "
                       "warm-up per precision",
           "unit": "instance-steps/s", "instances_per_N": {str(k): int((sizes == k).sum()) for k in sizes_all}}
    final = {}
    for prec in (64, 32):
        states = [x.clone() for x in Wf]
        for _ in range(warmup):
            qbgpu.homogeneous_batch(states, dt, 1, rk4=True, J=J, M=M, L=L, R=R, precision=prec)
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for k in range(steps):
            flush.zero_()
            evs[k][0].record()
            qbgpu.homogeneous_batch(states, dt, 1, rk4=True, J=J, M=M, L=L, R=R, precision=prec)
            evs[k][1].record()
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs) / steps
        out[f"f{prec}"] = {"value": round(ninst / (ms * 1e-3), 3), "ms_per_step": round(ms, 3)}
        final[prec] = torch.cat([x.reshape(-1) for x in states]).cpu().numpy()
    out["speedup_f32_vs_f64"] = round(out["f32"]["value"] / out["f64"]["value"], 4)
    out["rel_l2_f32_vs_f64_final_states"] = float(np.linalg.norm(final[32] - final[64]) / np.linalg.norm(final[64]))
    if args.config3_big > 0:
        # the configuration's instance count in the FP32 form
        nbig = args.config3_big
        sizes_b = rng.choice(sizes_all, size=nbig, p=w / w.sum())
        states = [qbgpu.to_fourier(torch.from_numpy(qbgpu.gaussian_mixture_state(int(n), L, seed=9000 + i, ncells=1)).cuda())[0].contiguous()
                  for i, n in enumerate(sizes_b)]
        qbgpu.homogeneous_batch(states, dt, 1, rk4=True, J=J, M=M, L=L, R=R, precision=32)     # tuning and sizing
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        e0.record()
        qbgpu.homogeneous_batch(states, dt, 2, rk4=True, J=J, M=M, L=L, R=R, precision=32)     # 2 direct steps
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 2
        out["f32_all_instances"] = {"instances": nbig, "instances_per_N": {str(k): int((sizes_b == k).sum()) for k in sizes_all},
                                    "value": round(nbig / (ms * 1e-3), 3), "ms_per_step": round(ms, 3),
                                    "timed": "2 RK4 steps in one call, after a first call that tuned and sized the groups"}
    out["schedules"] = [s_ for s_ in qbgpu.batch_schedules() if s_["J"] == J and s_["M"] == M]
    return out


def run_precision_form(args, wl, qbgpu, q, B, Wall, flush, value64):
    """The FP32 form of the collision operator on the same workload and timing
    protocol, with its error against the FP64 path: Cc and Cd of the initial
    state (relative L2 and L1 over all cells) and the state after the timed
    number of Strang steps (relative L1)."""
    import torch
    N, cells = wl["N"], wl["cells"]
    ws32, ws64 = qbgpu.Workspace(N, precision=32), qbgpu.Workspace(N)
    W0 = torch.from_numpy(Wall[:cells].copy()).cuda()
    bufs = [W0.clone(), torch.empty_like(W0)]

    def step(Win, Wout):
        qbgpu.inhom_step(ws32, q, Win, wl["h"], wl["dt"], B, out=Wout)
    for i in range(args.warmup):
        step(bufs[i % 2], bufs[(i + 1) % 2])
    torch.cuda.synchronize()
    ws32.i3_forms(reset=True)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    cur = args.warmup % 2
    for k in range(args.steps):
        flush.zero_()
        evs[k][0].record()
        step(bufs[cur], bufs[1 - cur])
        evs[k][1].record()
        cur = 1 - cur
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    value32 = cells * 2 * args.steps / (ms * 1e-3)
    real, total = ws32.i3_forms()      # cell evaluations of the timed steps, by I3 form

    def rel(a, b, o):
        a, b = a.cpu().numpy().ravel(), b.cpu().numpy().ravel()
        return float(np.linalg.norm(a - b, o) / np.linalg.norm(b, o))
    Wf = torch.empty((cells, 4, N, N), dtype=torch.complex128, device="cuda")
    qbgpu._check(qbgpu.lib().qb_to_fourier(N, 4 * cells, qbgpu._ptr(W0), qbgpu._ptr(Wf), qbgpu._stream()), "qb_to_fourier")
    cc64, cd64 = qbgpu.collision_operators(ws64, q, Wf)
    cc32, cd32 = qbgpu.collision_operators(ws32, q, Wf)
    a, b = W0.clone(), W0.clone()
    for _ in range(args.steps):
        a = qbgpu.inhom_step(ws64, q, a, wl["h"], wl["dt"], B)
        b = qbgpu.inhom_step(ws32, q, b, wl["h"], wl["dt"], B)
    # a long run on a few cells: the state after 1000 steps
    long_cells, long_steps = 8, 1000
    a8, b8 = W0[:long_cells].clone(), W0[:long_cells].clone()
    B8 = B[:long_cells].contiguous()
    na, nb = torch.empty_like(a8), torch.empty_like(b8)
    for _ in range(long_steps):
        qbgpu.inhom_step(ws64, q, a8, wl["h"], wl["dt"], B8, out=na)
        qbgpu.inhom_step(ws32, q, b8, wl["h"], wl["dt"], B8, out=nb)
        a8, na, b8, nb = na, a8, nb, b8
    torch.cuda.synchronize()
    return {"dtype": "f32 (FFTs, spectra, tables); f64 state, assembly and update", "value": round(value32, 3), "unit": UNIT,
            "ms_per_step": round(ms / args.steps, 4), "sim_steps_per_s": round(args.steps / (ms * 1e-3), 4),
            "speedup_vs_fp64": round(value32 / value64, 4), "i3_real_form_cells": f"{real} of {total}",
            "rel_err_vs_fp64": {"Cc_l2": rel(cc32, cc64, 2), "Cd_l2": rel(cd32, cd64, 2), "Cc_l1": rel(cc32, cc64, 1),
                                "Cd_l1": rel(cd32, cd64, 1), f"W_l1_after_{args.steps}_steps": rel(b, a, 1),
                                f"W_l1_after_{long_steps}_steps_first_{long_cells}_cells": rel(b8, a8, 1)},
            "bound": 1e-5}


def run_dftmma_sample(args, qbgpu, flush, cells=64, N=16, J=16, M=16, L=6.0, R=3.75):
    """The I3 sums of the FP32 form at N = 16 two ways: the FFT kernels
    (k_i3, 4-CTA clusters) and DFT-GEMMs on the tensor cores (k_i3_mma32:
    tcgen05.mma kind::tf32, TF32 hi/lo split); C[W] of `cells` cells per
    evaluation, both against the FP64 operator.  Tensor-pipe work: every
    1-D pass is a 128 x 64 x 64 real GEMM per 4 grids, 3 products (hi/lo)."""
    import torch
    import ctypes
    L_ = qbgpu.lib()
    q = qbgpu.Quad(N, J, M, L, R)
    W = qbgpu.to_fourier(torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=5, ncells=cells)).cuda())
    ws64 = qbgpu.Workspace(N)
    cc64, cd64 = qbgpu.collision_operators(ws64, q, W)

    def rel(a, b):
        return float(torch.linalg.norm((a - b).flatten()) / torch.linalg.norm(b.flatten()))
    out = {"workload": f"N={N} (padded {2 * N}), J={J}, M={M}, L={L}, R={R}, {cells} cells, FP32 form, C[W] of every cell "
                       f"per evaluation; {args.steps} timed evaluations after {args.warmup} warm-up per variant, L2 flushed",
           "unit": UNIT}
    for var, name in ((0, "fft_kernels"), (1, "tensor_core_dft_gemm")):
        ws = qbgpu.Workspace(N, precision=32)
        ws.set_i3_variant(var)
        for _ in range(args.warmup):
            qbgpu.collision_operators(ws, q, W)
        torch.cuda.synchronize()
        L_.qb_profile_reset()
        L_.qb_profile_enable(1)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record()
            cc, cd = qbgpu.collision_operators(ws, q, W)
            evs[k][1].record()
        torch.cuda.synchronize()
        L_.qb_profile_enable(0)
        ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
        kms, kn = ctypes.c_double(), ctypes.c_long()
        L_.qb_profile_read(b"i3_cluster", ctypes.byref(kms), ctypes.byref(kn))
        i3_ms = kms.value / max(1, kn.value)
        entry = {"value": round(cells / (ms * 1e-3), 3), "ms_per_eval": round(ms, 4), "i3_kernel_ms": round(i3_ms, 4),
                 "rel_l2_vs_fp64": {"Cc": rel(cc, cc64), "Cd": rel(cd, cd64)}, "device_errors": ws.device_errors()}
        if var == 1:
            passes = 2 + 4 * 4                                  # per (cell, term): spectra tile + 4 chain tiles x 4 passes
            flops = cells * J * M * passes * 3 * 2 * 128 * 64 * 64
            entry["tensor_flops_per_launch"] = flops
            entry["tensor_tflops"] = round(flops / (i3_ms * 1e-3) / 1e12, 3)
            entry["kernel"] = "k_i3_mma32 (tcgen05.mma kind::tf32, M128 N64 K8, accumulators in tensor memory)"
        out[name] = entry
    out["tensor_core_vs_fft_i3_kernel"] = round(out["fft_kernels"]["i3_kernel_ms"] / out["tensor_core_dft_gemm"]["i3_kernel_ms"], 4)
    return out


def run_surrogate(args, wl, qbgpu, q, B, Wall, flush, value64, nseeds=1024, samples=3, iters=8000, lr=5e-3):
    """The learned collision operator on the same workload and timing
    protocol.  A Fourier neural operator (width 32, 12 modes, 4 layers) is
    trained on (W, Cc + Cd) pairs of `nseeds` seeded mixture cells and their
    homogeneous relaxation (exact FP64 operator), each minibatch turned by
    random spin rotations (the operator commutes with them), then drives the collision
    half of the Strang steps: the exact operator judges every 10th step and
    takes over, until the next check, the cells whose collision increment from
    the network differed from the exact one by more than 0.5 (relative L1).  Reported: the rate, the training cost, the network's error
    on the workload's initial state, how many cell-steps each operator took,
    and the state's deviation from the FP64 run after the same steps."""
    import torch
    N, cells = wl["N"], wl["cells"]
    ws = qbgpu.Workspace(N)
    t0 = time.perf_counter()
    X, Y = qbgpu.relaxation_pairs(ws, q, torch.from_numpy(qbgpu.mixture_cells(N, wl["L"], nseeds, 5000)).cuda(), samples)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    net = qbgpu.FNO(N, width=32, modes=12, layers=4, seed=1)
    net.fit_scales(X, Y)
    t0 = time.perf_counter()
    loss = qbgpu.train_fno(net, X, Y, iters, batch=64, lr=lr, spin_rotations=True)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    del X, Y

    def rel(a, b):
        a, b = a.cpu().numpy().ravel(), b.cpu().numpy().ravel()
        return float(np.abs(a - b).sum() / np.abs(b).sum())
    W0 = torch.from_numpy(Wall[:cells].copy()).cuda()
    cc, cd = qbgpu.collision_operators(ws, q, qbgpu.to_fourier(W0))
    c_err = rel(net.forward(W0), qbgpu.from_fourier(cc + cd))
    tol, every = 0.5, 10
    sur = qbgpu.Surrogate(net, tol=tol, check_every=every)
    bufs = [W0.clone(), torch.empty_like(W0)]
    for i in range(args.warmup):
        sur.step(ws, q, bufs[i % 2], wl["h"], wl["dt"], B, out=bufs[(i + 1) % 2])
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    cur = args.warmup % 2
    for k in range(args.steps):
        flush.zero_()
        evs[k][0].record()
        sur.step(ws, q, bufs[cur], wl["h"], wl["dt"], B, out=bufs[1 - cur])
        evs[k][1].record()
        cur = 1 - cur
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    value = cells * 2 * args.steps / (ms * 1e-3)
    ns, ne, res = sur.stats()
    a = W0.clone()
    for _ in range(args.warmup + args.steps):
        a = qbgpu.inhom_step(ws, q, a, wl["h"], wl["dt"], B)
    torch.cuda.synchronize()
    long_run = surrogate_long_run(qbgpu, net, q, W0, wl, args.surrogate_long_steps, args.surrogate_long_cells) \
        if args.surrogate_long_steps > 0 else None
    # the trained network's inference with the pointwise maps and DFTs on the tensor cores (BF16, FP32 accumulation)
    infer = {}
    for tc in (False, True):
        net.set_tensor_cores(tc)
        for _ in range(3):
            yb = net.forward(W0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(20):
            yb = net.forward(W0)
        e1.record()
        torch.cuda.synchronize()
        infer["tensor_cores" if tc else "fp32"] = {"cells_per_s": round(cells * 20 / (e0.elapsed_time(e1) * 1e-3), 1), "out": yb.clone()}
    net.set_tensor_cores(False)
    tc_vs_fp32 = rel(infer["tensor_cores"].pop("out"), infer["fp32"].pop("out"))
    infer["rel_l1_tensor_cores_vs_fp32"] = round(tc_vs_fp32, 6)
    infer["device_errors"] = net.device_errors()
    return {"what": f"Strang steps with the collision half from a Fourier neural operator (FP32), exact FP64 operator as judge "
                    f"every {every}th step and per-cell fallback above a relative L1 difference {tol} of the collision increment; "
                    f"the checking steps are inside "
                    f"the timed region",
            "long_run": long_run,
            "value": round(value, 3), "unit": UNIT, "ms_per_step": round(ms / args.steps, 4),
            "speedup_vs_fp64": round(value / value64, 4),
            "training": {"pairs": nseeds * samples, "iterations": iters, "batch": 64, "lr": lr, "spin_rotations": True, "final_loss": loss,
                         "data_s": round(t_data, 2), "train_s": round(t_train, 2), "params": net.num_params},
            "C_rel_l1_on_initial_state": round(c_err, 5),
            "cell_steps": {"surrogate": ns, "exact": ne}, "last_max_residual": round(res, 5),
            f"W_rel_l1_vs_fp64_after_{args.warmup + args.steps}_steps": rel(bufs[cur], a),
            "inference_forward": infer}


def surrogate_long_run(qbgpu, net, q, W0, wl, steps, cells, tols=(0.5, 0.1, 0.02, 1e-5), every=10):
    """The surrogate's trajectory against the FP64 one over `steps` Strang
    steps of the first `cells` x-cells (a periodic line of them, the workload's
    h and dt), for judge tolerances `tols` (relative L1 of the collision
    increment; 1e-5 is the configuration's residual bound): deviation of W,
    cell-steps per operator, and the time per step against the FP64 step."""
    import torch
    N = wl["N"]
    Ws = W0[:cells].contiguous()
    B = torch.zeros((cells, 3), dtype=torch.float64, device="cuda")
    ws = qbgpu.Workspace(N)

    def run(step):
        a, b = Ws.clone(), torch.empty_like(Ws)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            step(a, b)
            a, b = b, a
        e1.record()
        torch.cuda.synchronize()
        return a, e0.elapsed_time(e1) / steps
    ref, ms64 = run(lambda a, b: qbgpu.inhom_step(ws, q, a, wl["h"], wl["dt"], B, out=b))
    out = {"what": f"{steps} Strang steps of the first {cells} x-cells (a periodic line of them), judge every {every} steps",
           "fp64_ms_per_step": round(ms64, 4), "by_tolerance": []}
    for tol in tols:
        sur = qbgpu.Surrogate(net, tol=tol, check_every=every)
        Wn, ms = run(lambda a, b: sur.step(ws, q, a, wl["h"], wl["dt"], B, out=b))
        ns, ne, _ = sur.stats()
        out["by_tolerance"].append({"tol": tol, "W_rel_l1_vs_fp64": float((Wn - ref).abs().sum() / ref.abs().sum()),
                                    "cell_steps": {"surrogate": ns, "exact": ne}, "ms_per_step": round(ms, 4),
                                    "speedup_vs_fp64": round(ms64 / ms, 4)})
    return out


def run_surrogate64(args, qbgpu, flush, cells=64, nseeds=1024, samples=3, iters=8000, lr=5e-3, steps=10, warmup=3):
    """The learned collision operator at N = 64 (the shape of the surrogate
    configuration: J = M = 32, FNO of 4 layers, width 32, 12 modes), on `cells`
    of a 4096-cell periodic domain (h = 1/4096).  Training pairs and the judge
    use the FP32 form of the exact operator (its C error against FP64 is about
    1e-6); the plain FP64 Strang step is timed alike for the ratio.  The exact
    operator judges every 10th step and takes over the cells whose collision
    increment from the network differed from the exact one by more than 0.5
    (relative L1) until the next check."""
    import torch
    N, J, M, L, R = 64, 32, 32, 6.0, 3.75
    h = 1.0 / 4096
    dt = 0.4 * h / L
    q = qbgpu.Quad(N, J, M, L, R)
    ws32, ws64 = qbgpu.Workspace(N, precision=32), qbgpu.Workspace(N)
    t0 = time.perf_counter()
    X, Y = qbgpu.relaxation_pairs(ws32, q, torch.from_numpy(qbgpu.mixture_cells(N, L, nseeds, 7000)).cuda(), samples)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    net = qbgpu.FNO(N, width=32, modes=12, layers=4, seed=1)
    net.fit_scales(X, Y)
    t0 = time.perf_counter()
    loss = qbgpu.train_fno(net, X, Y, iters, batch=64, lr=lr, spin_rotations=True)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    del X, Y

    def rel(a, b):
        a, b = a.cpu().numpy().ravel(), b.cpu().numpy().ravel()
        return float(np.abs(a - b).sum() / np.abs(b).sum())
    W0 = torch.from_numpy(qbgpu.gaussian_mixture_state(N, L, seed=4, ncells=cells)).cuda()
    B = torch.zeros((cells, 3), dtype=torch.float64, device="cuda")
    cc, cd = qbgpu.collision_operators(ws64, q, qbgpu.to_fourier(W0))
    c_err = rel(net.forward(W0), qbgpu.from_fourier(cc + cd))

    def timed(stepfn, n, w):
        bufs = [W0.clone(), torch.empty_like(W0)]
        for i in range(w):
            stepfn(bufs[i % 2], bufs[(i + 1) % 2])
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        cur = w % 2
        for k in range(n):
            flush.zero_()
            evs[k][0].record()
            stepfn(bufs[cur], bufs[1 - cur])
            evs[k][1].record()
            cur = 1 - cur
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs) / n, bufs[cur]
    ms64, W64 = timed(lambda a, b: qbgpu.inhom_step(ws64, q, a, h, dt, B, out=b), 2, 1)
    tol, every = 0.5, 10
    sur = qbgpu.Surrogate(net, tol=tol, check_every=every)
    ms_sur, Wsur = timed(lambda a, b: sur.step(ws32, q, a, h, dt, B, out=b), steps, warmup)
    ns, ne, res = sur.stats()
    a = W0.clone()
    for _ in range(warmup + steps):
        a = qbgpu.inhom_step(ws64, q, a, h, dt, B)
    torch.cuda.synchronize()
    return {"workload": f"N={N} (padded {2 * N}), J={J}, M={M}, {cells} of 4096 x-cells, h=1/4096, dt=0.4h/L, periodic; "
                        f"FNO width 32, 12 modes, 4 layers; judge: FP32 form of the exact operator every {every}th step "
                        f"(inside the timed region), per-cell fallback above a relative L1 difference {tol} of the collision increment",
            "unit": UNIT, "fp64": {"value": round(cells * 2 / (ms64 * 1e-3), 3), "ms_per_step": round(ms64, 3)},
            "surrogate": {"value": round(cells * 2 / (ms_sur * 1e-3), 3), "ms_per_step": round(ms_sur, 3)},
            "speedup_vs_fp64": round(ms64 / ms_sur, 3),
            "training": {"pairs": nseeds * samples, "data": "FP32 form", "iterations": iters, "batch": 64, "lr": lr,
                         "spin_rotations": True, "final_loss": loss, "data_s": round(t_data, 2), "train_s": round(t_train, 2)},
            "C_rel_l1_on_initial_state": round(c_err, 5), "cell_steps": {"surrogate": ns, "exact": ne},
            "last_max_residual": round(res, 5), f"W_rel_l1_vs_fp64_after_{warmup + steps}_steps": rel(Wsur, a)}


def run_e2e(args, wl, qbgpu, qd, world, rank, q, ws, B, Wall):
    import torch
    N, cells = wl["N"], wl["cells"]
    steps = max(1, min(args.steps, 5))
    nbytes = cells * 4 * N * N * 8
    if world == 1 and N == qbgpu.N_GRID:
        up = qbgpu.Upstream()
        quads = [up.fourier(1, wl["J"], wl["L"], wl["R"]), up.fourier(2, wl["J"], wl["L"], wl["R"]),
                 up.fourier(3, wl["J"], wl["L"], wl["R"], wl["M"]), up.fourier(4, wl["J"], wl["L"], wl["R"])]
        it = up.inhom_interm(cells, wl["L"])
        hin = torch.from_numpy(Wall[:cells].copy()).pin_memory().numpy()
        hout = torch.empty(hin.shape, dtype=torch.float64).pin_memory().numpy()
        hB = torch.zeros((cells, 3), dtype=torch.float64).pin_memory().numpy()
        up.inhom_step(hin, quads, wl["h"], wl["dt"], hB, L=wl["L"], interm=it)      # warm-up
        t0 = time.perf_counter()
        a, b = hin, hout
        for _ in range(steps):
            up.inhom_step(a, quads, wl["h"], wl["dt"], hB, L=wl["L"], interm=it, out=b)
            a, b = b, a
        wall = time.perf_counter() - t0
        up.L.InhomStepInterm_Delete(qbgpu.C.byref(it))
        for w, qq in zip((1, 2, 3, 4), quads):
            up.quad_delete(w, qq)
        return {"value": round(cells * 2 * steps / wall, 3), "unit": UNIT, "h2d_bytes_per_step": nbytes + cells * 3 * 8,
                "d2h_bytes_per_step": nbytes, "api": "InhomStepPeriodic (upstream C API, host buffers, pinned)", "steps": steps}
    # sharded path with host staging per step, device-timed (CUDA events on
    # the stream that carries the copies and kernels), max over ranks
    hin = torch.from_numpy(Wall[rank * cells:(rank + 1) * cells].copy()).pin_memory()
    hout = torch.empty_like(hin).pin_memory()

    sharded = None
    if world > 1:
        sharded = qd.ShardedStrang(cells, (4, N, N), torch.float64, "cuda",
                                   lambda ext, out: qbgpu.transport(ext, wl["L"], wl["h"], 0.5 * wl["dt"], out=out),
                                   lambda c, i: qbgpu.fourier_collision(ws, q, c, wl["dt"], B[i:i + c.shape[0]]))
    import torch.distributed as dist
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        Wd = hin.cuda(non_blocking=True)
        if world > 1:
            Wn = sharded.step(Wd)
        else:
            Wn = qbgpu.inhom_step(ws, q, Wd, wl["h"], wl["dt"], B)
        hout.copy_(Wn, non_blocking=True)
        hin, hout = hout, hin
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return {"value": round(world * cells * 2 * steps / (ms * 1e-3), 3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes, "api": "sharded Strang step (qbgpu batched API + NCCL halos), host staging, device-timed",
            "steps": steps}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = workload(args)
    kind = ref_kind()
    if kind is None:
        print(json.dumps({"impl": "reference", "unavailable": "upstream sources were not compiled into oracle/_ref (no checkout at build time)"}))
        return
    procs = max(1, min(os.cpu_count() or 1, args.cpu_procs))
    for i in range(args.warmup):
        cpu_sample(wl, procs, seed_offset=i)
    rates, walls = [], []
    for k in range(args.steps):
        r, w = cpu_sample(wl, procs, seed_offset=args.warmup + k)
        rates.append(r)
        walls.append(w)
    total = sum(walls)
    value = procs * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian mixture)",
            "config": config_json(wl, 1, "n/a (CPU)"),
            "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": procs, "kind": kind,
                             "sample": f"per step {procs} processes x 1 cell-collision evaluation (CcInt + CdInt) of the upstream C "
                                       f"sources; FFTs through the project's CPU FFTW-API shim (FFTW absent)"},
            "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cells", type=int, default=64)
    ap.add_argument("--grid", type=int, default=32)
    ap.add_argument("--J", type=int, default=16)
    ap.add_argument("--M", type=int, default=16)
    ap.add_argument("--cpu-procs", type=int, default=min(32, os.cpu_count() or 1))
    ap.add_argument("--no-precision-form", action="store_true", help="skip the FP32-form measurement")
    ap.add_argument("--no-config2", action="store_true", help="skip the N = 64 precision-form sample")
    ap.add_argument("--config2-cells", type=int, default=64, help="x-cells of the N = 64 sample (of its 1024)")
    ap.add_argument("--config2-long-steps", type=int, default=1000,
                    help="Strang steps of the N = 64 FP32-against-FP64 long run (0 skips it)")
    ap.add_argument("--config2-long-cells", type=int, default=2, help="x-cells of the N = 64 long run")
    ap.add_argument("--no-config3", action="store_true", help="skip the mixed-size batch sample")
    ap.add_argument("--config3-big", type=int, default=4096,
                    help="instances of the FP32 mixed-size batch at the configuration's count (0 skips it)")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the learned-operator measurement")
    ap.add_argument("--surrogate-n64", action="store_true", help="add the learned operator at N = 64 (about two minutes)")
    ap.add_argument("--surrogate-long-steps", type=int, default=1000,
                    help="Strang steps of the surrogate-against-FP64 long run (0 skips it)")
    ap.add_argument("--surrogate-long-cells", type=int, default=16, help="x-cells of the surrogate long run")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-dftmma", action="store_true", help="skip the tensor-core DFT-GEMM sample (N = 16)")
    ap.add_argument("--config3-only", action="store_true",
                    help="print only the mixed-size batch sample (a small case for profiling, with --config3-ninst)")
    ap.add_argument("--config3-ninst", type=int, default=256, help="instances of the mixed-size batch sample")
    ap.add_argument("--config3-sizes", default="", help="comma-separated subset of the sizes of the batch sample")
    ap.add_argument("--dftmma-only", action="store_true",
                    help="run only the tensor-core DFT-GEMM sample and print its JSON block (for profiling)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    elif args.dftmma_only:
        import torch
        qbgpu = _import("qbgpu", os.path.join(PKG, "qbgpu.py"))
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
        print(json.dumps(run_dftmma_sample(args, qbgpu, flush)), flush=True)
    elif args.config3_only:
        import torch
        qbgpu = _import("qbgpu", os.path.join(PKG, "qbgpu.py"))
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
        print(json.dumps(run_config3_sample(args, qbgpu, flush, ninst=args.config3_ninst)), flush=True)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
