#!/usr/bin/env python
"""FDTD throughput benchmark: Mcell-updates/s of the Yee step loop on one B200 per rank.

Workload (default): 512^3 cells (513^3 = 135,005,697 nodes), 1 mm cells, 10-cell CPML, 200
seeded random dielectric spheres (radius 5-40 cells, eps_r U[1,10], sigma U[0,0.05] S/m), 20 % of
them one-pole Debye (delta eps U[1,5], one seeded tau in [5,50] ps), one 50-ohm port driven by a
Gaussian pulse (f0 10 GHz, fc 5 GHz). A step is one time step over the whole grid (fused E+H march,
Debye ADE, source, port V/I probe). Fields are 6.5 GB per buffer set, far larger than the 126 MB
L2, so no flush is needed between timed steps.

value: whole-job nodes x steps / device time of the K timed steps (CUDA events on the session's
stream, max over ranks). Ranks run independent replicas (weak scaling): the reference solves one
grid on one device, and this engine keeps a grid on one GPU.

--impl reference: the CPU baseline arm (rank 0 only): the oracle (a C++ restatement of the
reference's own CPU FDTD, cpu.rs) on all host cores, on a bounded sample of full time steps of the
same grid.
"""
from __future__ import annotations

import argparse
import copy
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

BYTES_PER_NODE = 48  # read + write of Ex Ey Ez Hx Hy Hz, f32


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The largest of every rank's x (a job's time is its slowest rank's); x itself at N = 1."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(nodes_per_rank: int, steps: int, world: int, ms_max: float) -> float:
    """Whole-job Mcell-updates/s of replicas: every rank's nodes x steps over the slowest rank's time."""
    return world * nodes_per_rank * steps / (ms_max / 1e3) / 1e6


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--cells", type=int, default=512, help="cells per axis (512 is the benchmark workload)")
    p.add_argument("--spheres", type=int, default=None, help="spheres in the grid (default: 200 at 256 cells and up)")
    p.add_argument("--separate", action="store_true", help="time the unfused H and E kernels instead")
    p.add_argument("--pml", type=int, default=None, help="CPML depth in cells (default: 10 at 512^3)")
    p.add_argument("--cpu-steps", type=int, default=8, help="full time steps the CPU baseline times")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="throughput: skip the batched and adjoint ratios that the line also carries")
    p.add_argument("--workload", choices=["throughput", "adjoint", "batched", "batched-adjoint", "antenna"],
                   default="throughput",
                   help="throughput: the 512^3 spheres step (the headline); adjoint: the flux-objective "
                        "gradient over a 32x32x8 design block on 160x160x96 cells, 4000 steps; batched: 192 "
                        "grids of U{48..160}^3 cells stepped together vs one after another, 1500 steps; "
                        "batched-adjoint: the same grids with a 16^3 design block each, their flux gradients "
                        "together vs one after another; antenna: the 256x256x192 patch antenna with its NTFF box at "
                        "3 frequencies, 6000 steps, and its far field")
    p.add_argument("--count", type=int, default=192, help="batched: grids in the batch")
    p.add_argument("--group", type=int, default=16, help="batched-adjoint: gradients in flight together")
    p.add_argument("--checkpoints", type=int, default=64, help="adjoint: field checkpoints (0: keep the history)")
    p.add_argument("--fd", type=int, default=32,
                   help="adjoint: parameters checked against central differences of the FP64 device forward")
    return p.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except Exception:
        return 6650.0, "profiling recipe fallback 6.65 TB/s (of fallback)"


def workload(cells: int, steps: int, fused: bool = True, pml=None, spheres=None):
    from fieldgrid_b200 import workloads as W
    if pml is None:
        pml = 10 if cells >= 256 else max(4, cells // 16)
    count = spheres if spheres is not None else (200 if cells >= 256 else max(8, cells // 3))
    rmin, rmax = (5, 40) if cells >= 256 else (2, max(3, cells // 12))
    return W.spheres(cells=cells, pml=pml, steps=steps, count=count, rmin=rmin, rmax=rmax, fused=fused)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str):
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")
        self.proc = None
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", device_id, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
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
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 8:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[4 + q].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def device_id(local_rank: int) -> str:
    try:
        import torch
        u = str(torch.cuda.get_device_properties(local_rank).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v for v in vis.split(",") if v.strip()]
        return ids[local_rank] if local_rank < len(ids) else str(local_rank)


def traffic_for(variant: str, workload_name: str):
    """DRAM bytes per launch of the dominant kernel from a committed ncu capture, when one exists
    for this kernel variant and workload."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        e = d.get(variant, {}).get(workload_name)
        return None if e is None else float(e)
    except Exception:
        return None


def run_reference(args):
    """The CPU arm: the oracle's State::step on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    sc = workload(args.cells, args.steps + args.warmup)
    n = sc.grid.dims()
    nn = n[0] * n[1] * n[2]
    t = time.time()
    osim = O.OracleSim(*sc.args(), bits=32)
    setup_s = time.time() - t
    k = max(1, min(args.steps, args.cpu_steps))
    w = max(1, min(args.warmup, 1))
    sec = O.time_steps(osim, 0, sc.pulse, sc.extras, w, k)
    value = nn * k / sec / 1e6
    cores = O.threads()
    line = {
        "impl": "reference", "metric": "Mcell-updates/s", "value": value, "unit": "Mcell/s", "n_gpus": args.gpus,
        "steps": k, "warmup": w, "ms_per_step": 1e3 * sec / k, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": sc.name, "nodes": nn, "cells": sc.grid.cells(), "setup_s": round(setup_s, 2)},
        "cpu_baseline": {"value": value, "unit": "Mcell/s", "cores": cores, "kind": "port",
                         "sample": f"{k} full time steps of the {n[0]}x{n[1]}x{n[2]}-node grid after {w} warm-up "
                                   f"step(s); C++ restatement of cpu.rs, OpenMP over x-planes"},
        "e2e": {"value": value, "unit": "Mcell/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline(args, sc):
    from oracle import oracle as O
    n = sc.grid.dims()
    nn = n[0] * n[1] * n[2]
    osim = O.OracleSim(*sc.args(), bits=32)
    k = max(1, args.cpu_steps)
    sec = O.time_steps(osim, 0, sc.pulse, sc.extras, 1, k)
    del osim
    return {"value": nn * k / sec / 1e6, "unit": "Mcell/s", "cores": O.threads(), "kind": "port",
            "sample": f"{k} full time steps of the {n[0]}x{n[1]}x{n[2]}-node grid after 1 warm-up step; "
                      f"C++ restatement of the reference's CPU FDTD (cpu.rs), OpenMP over x-planes"}


def run_adjoint(args):
    """The adjoint workload: time of the gradient (forward with checkpoints + segment recomputation
    + backward sweep) over the time of a plain forward of the same run, device-timed per phase, and
    wall-clock through the public call (fdtd.flux_gradient) with host buffers."""
    import numpy as np
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    from fieldgrid_b200 import fdtd
    from fieldgrid_b200 import workloads as W
    from fieldgrid_b200.gpu import Gpu, Options
    g = Gpu.open(Options(device=torch.cuda.current_device()))
    scene, spec, _, _ = W.flux_design(steps=args.steps if args.steps != 2000 else 4000, checkpoints=args.checkpoints)
    sc = scene()
    sim = fdtd.Sim.try_new(*sc.args())
    fwd, grad = [], []
    sampler = None
    for rep in range(max(args.warmup, 3) + 3):
        timed = rep >= max(args.warmup, 3)
        if timed and sampler is None:
            sampler = ClockSampler(device_id(int(os.environ.get("LOCAL_RANK", "0"))))
        t = time.perf_counter()
        f = fdtd.flux_gradient(g, sim, 0, sc.pulse, spec, grad=False)
        tf = time.perf_counter() - t
        t = time.perf_counter()
        r = fdtd.flux_gradient(g, sim, 0, sc.pulse, spec, grad=True)
        tg = time.perf_counter() - t
        if timed:
            fwd.append((tf, f.forward_ms))
            grad.append((tg, r))
    clocks = sampler.stop()
    # central differences (h = 1e-4) of the FP64 device forward on seeded parameters (seed 5)
    fd = None
    if args.fd > 0 and rank == 0:
        r = grad[-1][1]
        _, _, eps0, sig0 = W.flux_design(steps=spec.steps, checkpoints=args.checkpoints)
        spec64 = fdtd.FluxSpec(spec.design_lo, spec.design_hi, spec.plane_k, spec.freq, spec.steps, precision=64)
        rng = W.SplitMix64(5)
        errs, t0 = [], time.perf_counter()
        for q in range(args.fd):
            at = tuple(rng.integer(0, n - 1) for n in spec.shape())
            which = "eps" if q % 2 == 0 else "sigma"
            base = eps0 if which == "eps" else sig0
            up, dn = base.copy(), base.copy()
            up[at] = np.float32(base[at] + 1e-4)
            dn[at] = np.float32(base[at] - 1e-4)
            h_eff = 0.5 * (float(up[at]) - float(dn[at]))   # the step the f32 materials carry
            js = []
            for arr in (up, dn):
                s2 = scene(*((arr, sig0) if which == "eps" else (eps0, arr)))
                js.append(fdtd.flux_gradient(g, fdtd.Sim.try_new(*s2.args()), 0, s2.pulse, spec64, grad=False).objective)
            fdv = (js[0] - js[1]) / (2 * h_eff)
            adj = float((r.grad_eps if which == "eps" else r.grad_sigma)[at])
            errs.append(abs(adj - fdv) / max(abs(fdv), 1e-300))
        fd = {"parameters": args.fd, "h": 1e-4, "reference": "FP64 forward on the device, central differences",
              "max_rel_err": float(max(errs)), "median_rel_err": float(np.median(errs)),
              "within_1e-3": int(sum(e <= 1e-3 for e in errs)), "seconds": time.perf_counter() - t0}
    if rank != 0:
        return None
    dev_f = float(np.median([x[1] for x in fwd]))
    dev_g = float(np.median([x[1].forward_ms + x[1].backward_ms for x in grad]))
    wall_f = float(np.median([x[0] for x in fwd]))
    wall_g = float(np.median([x[0] for x in grad]))
    r = grad[-1][1]
    line = {
        "metric": "adjoint grad time / forward", "value": dev_g / dev_f, "unit": "x", "n_gpus": world,
        "steps": spec.steps, "warmup": max(args.warmup, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": sc.name, "cells": [160, 160, 96], "design_cells": spec.cells(),
                   "parameters": 2 * spec.cells(), "checkpoints": args.checkpoints, "segments": r.segments,
                   "segment_len": r.segment_len, "design_edges": r.design_edges, "freq_hz": spec.freq},
        "forward_ms": dev_f, "gradient_ms": dev_g,
        "gradient_parts_ms": {"forward": r.forward_ms, "backward": r.backward_ms, "recompute_device": r.recompute_ms,
                              "sweep_device": r.adjoint_ms},
        "e2e": {"value": wall_g / wall_f, "unit": "x", "forward_s": wall_f, "gradient_s": wall_g,
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "run": "fdtd.flux_gradient wall clock: setup of the session, the steps, read-back of the plane and "
                       "the gradient"},
        "objective": r.objective, "clocks": clocks, "fd_check": fd,
    }
    return line


def run_antenna(args):
    """The antenna workload: the patch antenna of 256x256x192 cells (12-cell CPML, PEC ground and
    patch on a 2-cell substrate, one 50-ohm port) with the near-to-far-field box 3 cells inside the
    CPML accumulating at 8, 10 and 12 GHz, all 6000 steps device-timed; then the far field on the
    5-degree theta/phi grid at each frequency (f64, device), and one fg_run of the same steps on
    host buffers (pack, upload, steps, read-back of the series and NTFF accumulators)."""
    import numpy as np
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    from fieldgrid_b200 import fdtd
    from fieldgrid_b200 import workloads as W
    from fieldgrid_b200.gpu import Gpu, Options
    g = Gpu.open(Options(device=local))
    K = args.steps if args.steps != 2000 else 6000
    Wm = max(args.warmup, 3)
    kt_steps = 10
    sc = W.patch_antenna(steps=Wm + K + kt_steps)
    sim = fdtd.Sim.try_new(*sc.args())
    pt = fdtd.patches(sim, sc.info["ntff_inset"])
    sc.extras.ntff = pt.gpu
    n = sim.dims()
    nn = n[0] * n[1] * n[2]
    s = fdtd.Session(g, sim, 0, sc.pulse, sc.extras)
    stream = torch.cuda.ExternalStream(s.stream)
    s.step(Wm)
    s.sync()
    sampler = ClockSampler(device_id(local))
    time.sleep(0.3)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    s.step(K)
    ev1.record(stream)
    ev1.synchronize()
    clocks = sampler.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    kt = s.kernel_times(kt_steps)
    launches = s.launches_per_step
    variant = s.variant
    s.close()
    field_parts = [k for k in ("fused_step", "shell_h", "shell_e", "update_h", "update_e") if k in kt]
    dom_ms = sum(kt[k] for k in field_parts)
    total_kt = sum(kt.values())
    peak, peak_src = measured_peaks()
    achieved = BYTES_PER_NODE * nn / (dom_ms / 1e3) / 1e9
    # the far field of the accumulated box on the 5-degree grid (37 x 72 directions), per frequency
    ex = copy.copy(sc.extras)
    ex.max_steps = K
    t0 = time.perf_counter()
    rec = fdtd.run(g, sim, 0, sc.pulse, ex)
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(time.perf_counter() - t0, world)
    th = np.deg2rad(np.arange(0, 181, 5, dtype=np.float64))
    ph = np.deg2rad(np.arange(0, 360, 5, dtype=np.float64))
    T, P = np.meshgrid(th, ph, indexing="ij")
    dirs = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3)
    nf = len(sc.extras.freqs)
    t0 = time.perf_counter()
    peaks = []
    for k, f in enumerate(sc.extras.freqs):
        far = fdtd.Far.load(pt, rec.ntff, nf, k, f, gpu=g)
        peaks.append(float(far.intensities(dirs).max()))
    far_ms = (time.perf_counter() - t0) * 1e3
    if rank != 0:
        return None
    return {
        "metric": "Mcell-updates/s", "value": job_rate(nn, K, world, ms), "unit": "Mcell/s", "n_gpus": world,
        "steps": K, "warmup": Wm, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": sc.name + ", NTFF box at 8/10/12 GHz", "nodes": nn, "pml": sc.info["pml"],
                   "patches": int(len(pt.area)), "freqs": list(sc.extras.freqs), "variant": variant,
                   "launches_per_step": launches},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "kernel": "field_update", "kernels": field_parts, "kernel_ms": dom_ms, "peak_source": peak_src},
        "kernel_ms": {k: round(v, 5) for k, v in kt.items()},
        "kernel_share": {k: round(v / total_kt, 4) for k, v in kt.items()},
        "ntff_share": round(kt.get("ntff", 0.0) / total_kt, 4),
        "gpu_launches": launches * K,
        "clocks": clocks,
        "e2e": {"value": job_rate(nn, K, world, t_e2e * 1e3), "unit": "Mcell/s", "h2d_bytes_per_step": rec.h2d / K,
                "d2h_bytes_per_step": rec.d2h / K,
                "run": f"one fg_run of {K} steps on host buffers: pack + upload, the steps, read-back of the series "
                       f"and the NTFF accumulators; wall clock"},
        "far_field": {"directions": int(len(dirs)), "freqs": nf, "ms": far_ms, "peak_intensity": peaks},
    }


def run_batched(args):
    """The batched workload: the same grids stepped one after another (a session per grid, its
    graphs, the TMA march where a clean box exists) and together (one batch); device-timed
    (CUDA events on each stream) over all steps; value = sequential time / batched time."""
    import numpy as np
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    from fieldgrid_b200 import fdtd
    from fieldgrid_b200 import workloads as W
    from fieldgrid_b200.gpu import Gpu, Options
    g = Gpu.open(Options(device=torch.cuda.current_device()))
    K = args.steps if args.steps != 2000 else 1500
    scenes = W.batch_grids(count=args.count, steps=K)
    t = time.perf_counter()
    sims = [fdtd.Sim.try_new(*sc.args()) for sc in scenes]
    t_setup = time.perf_counter() - t
    nodes = [int(np.prod(sc.grid.dims())) for sc in scenes]
    total = float(sum(nodes))
    sampler = ClockSampler(device_id(int(os.environ.get("LOCAL_RANK", "0"))))
    # one after another: each grid's own session and graphs
    seq_ms = 0.0
    for sc, sim in zip(scenes, sims):
        s = fdtd.Session(g, sim, 0, sc.pulse, sc.extras)
        s.step(2)
        s.sync()
        stream = torch.cuda.ExternalStream(s.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step(K)
        e1.record(stream)
        e1.synchronize()
        seq_ms += e0.elapsed_time(e1)
        s.close()
    # together
    t = time.perf_counter()
    b = fdtd.Batch(g, sims, [sc.pulse for sc in scenes], K + 2, tune=True)
    t_tune = time.perf_counter() - t
    b.step(2)
    b.sync()
    t0 = time.perf_counter()
    b.step(K)
    b.sync()
    bat_ms = (time.perf_counter() - t0) * 1e3
    info = b.info()
    series = [b.read(q, "series", (K + 2) * 2) for q in range(min(4, len(scenes)))]
    b.close()
    clocks = sampler.stop()
    if rank != 0:
        return None
    line = {
        "metric": "batched speed-up over sequential per-grid runs", "value": seq_ms / bat_ms, "unit": "x",
        "n_gpus": world, "steps": K, "warmup": 2, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{len(scenes)} grids U{{48..160}}^3 cells (multiples of 8), 8-cell CPML, "
                               f"random spheres (20% Debye), one point source each", "grids": len(scenes),
                   "nodes_total": int(total), "nodes_min": min(nodes), "nodes_max": max(nodes)},
        "batched_ms": bat_ms, "sequential_ms": seq_ms,
        "batched_mcells": total * K / (bat_ms / 1e3) / 1e6, "sequential_mcells": total * K / (seq_ms / 1e3) / 1e6,
        "tuned": info, "tune_s": t_tune, "setup_s": t_setup,
        "timing": "sequential: CUDA events around each grid's steps on its stream, summed; batched: wall clock "
                  "around the graph launches after a sync (one stream)",
        "clocks": clocks,
        "series_finite": bool(all(np.all(np.isfinite(x)) for x in series)),
    }
    return line


def run_batched_adjoint(args):
    """The batched workload's adjoint variant: each grid with a 16^3 design block and a flux
    objective, its gradient taken one grid after another (fdtd.flux_gradient per grid) and for all
    grids at once (fdtd.flux_gradient_batch, 16 runs in flight); wall clock around each, setup of
    the device sessions included in both; value = sequential time / batched time."""
    import numpy as np
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    from fieldgrid_b200 import fdtd
    from fieldgrid_b200 import workloads as W
    from fieldgrid_b200.gpu import Gpu, Options
    g = Gpu.open(Options(device=torch.cuda.current_device()))
    K = args.steps if args.steps != 2000 else 1500
    ck = args.checkpoints if args.checkpoints != 64 else int(round(K ** 0.5))
    jobs = W.batch_flux(count=args.count, steps=K, checkpoints=ck)
    scenes = [j[0]() for j in jobs]
    sims = [fdtd.Sim.try_new(*sc.args()) for sc in scenes]
    specs = [j[1] for j in jobs]
    pulses = [sc.pulse for sc in scenes]
    nodes = [int(np.prod(sc.grid.dims())) for sc in scenes]
    # warm-up: the first two runs both ways
    fdtd.flux_gradient_batch(g, sims[:2], pulses[:2], specs[:2], group=args.group)
    for q in range(2):
        fdtd.flux_gradient(g, sims[q], 0, pulses[q], specs[q])
    sampler = ClockSampler(device_id(int(os.environ.get("LOCAL_RANK", "0"))))
    t = time.perf_counter()
    seq = [fdtd.flux_gradient(g, sim, 0, p, spec) for sim, p, spec in zip(sims, pulses, specs)]
    seq_s = time.perf_counter() - t
    t = time.perf_counter()
    bat = fdtd.flux_gradient_batch(g, sims, pulses, specs, group=args.group)
    bat_s = time.perf_counter() - t
    clocks = sampler.stop()
    same = all(a.objective == b.objective and np.array_equal(a.grad_eps, b.grad_eps) and
               np.array_equal(a.grad_sigma, b.grad_sigma) for a, b in zip(seq, bat))
    if rank != 0:
        return 0
    line = {
        "metric": "batched adjoint speed-up over sequential per-grid gradients", "value": seq_s / bat_s, "unit": "x",
        "n_gpus": world, "steps": K, "warmup": 2, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{len(jobs)} grids U{{48..160}}^3 cells (multiples of 8), 8-cell CPML, random "
                               f"spheres (20% Debye), a 16^3 design block and a flux plane each", "grids": len(jobs),
                   "nodes_total": int(sum(nodes)), "checkpoints": ck, "group": args.group},
        "batched_s": bat_s, "sequential_s": seq_s, "results_equal": bool(same),
        "sequential_setup_s": sum(r.setup_ms for r in seq) / 1e3,
        "sequential_forward_backward_s": sum(r.forward_ms + r.backward_ms for r in seq) / 1e3,
        "batched_setup_s": sum(r.setup_ms for r in bat) / 1e3,
        "timing": "wall clock around all gradients (sessions set up inside both)",
        "clocks": clocks,
    }
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload in ("adjoint", "batched", "antenna"):
        line = {"adjoint": run_adjoint, "batched": run_batched, "antenna": run_antenna}[args.workload](args)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0
    if args.workload == "batched-adjoint":
        return run_batched_adjoint(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and "OMP_NUM_THREADS" not in os.environ:
        os.environ["OMP_NUM_THREADS"] = str(max(1, (os.cpu_count() or 8) // world))
    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))

    from fieldgrid_b200 import fdtd
    from fieldgrid_b200.gpu import Gpu, Options

    K, W = args.steps, max(args.warmup, 3)
    kt_steps = 10
    t = time.time()
    sc = workload(args.cells, W + K + kt_steps + (48 if K >= 48 else 0), fused=not args.separate, pml=args.pml,
                  spheres=args.spheres)
    t_mat = time.time() - t
    t = time.time()
    sim = fdtd.Sim.try_new(*sc.args())
    t_setup = time.time() - t
    n = sim.dims()
    nn = n[0] * n[1] * n[2]
    g = Gpu.open(Options(device=local))
    t = time.time()
    s = fdtd.Session(g, sim, 0, sc.pulse, sc.extras)
    t_session = time.time() - t
    log(f"rank {rank}: {sc.name}, {nn} nodes, classes {sim.coef_classes()}, debye edges {sim.count('debye_edges')}, "
        f"materials {t_mat:.1f}s setup {t_setup:.1f}s upload {t_session:.2f}s, {s.variant}")
    stream = torch.cuda.ExternalStream(s.stream)
    s.step(W)
    if K >= 48:
        # the two-step mode captures its 48-step graph for a step phase (t mod 6) on first use:
        # 48 more warm-up steps capture it for the phase the timed steps start at
        s.step(48)
        W += 48
    s.sync()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(device_id(local))
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    s.step(K)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, world)
    value = job_rate(nn, K, world, ms_max)

    # per-kernel device times of the same step (events between eager launches)
    kt = s.kernel_times(kt_steps)
    launches = s.launches_per_step
    energy = s.energy()
    variant = s.variant
    classes = sim.coef_classes()
    debye_edges = sim.count("debye_edges")
    s.close()
    # the field update of a step: the march over the clean box plus the CPML shell kernels (or the
    # separate H and E kernels; in the two-step mode half a two-step march plus the one-step march
    # of the remaining tiles and the shell, per step); its time is what the 48 B/node roofline is
    # measured against
    field_parts = [k for k in ("two_step", "edge_step", "fused_step", "shell_h", "shell_e", "update_h", "update_e")
                   if k in kt]
    dom_name, dom_ms = "field_update", sum(kt[k] for k in field_parts)
    peak, peak_src = measured_peaks()
    achieved = BYTES_PER_NODE * nn / (dom_ms / 1e3) / 1e9
    total_kt = sum(kt.values())

    e2e = None
    if not args.no_e2e:
        ex = copy.copy(sc.extras)
        ex.max_steps = K
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        rec = fdtd.run(g, sim, 0, sc.pulse, ex)
        torch.cuda.synchronize()
        t_e2e = time.perf_counter() - t0
        t_e2e = max_over_ranks(t_e2e, world)
        e2e = {"value": job_rate(nn, K, world, t_e2e * 1e3), "unit": "Mcell/s",
               "h2d_bytes_per_step": rec.h2d / K, "d2h_bytes_per_step": rec.d2h / K,
               "run": f"one fg_run of {K} steps on host buffers: pack + upload of the grid, the steps, energy checks "
                      f"every {ex.check_every or 1000}, read-back of the series; wall clock, max over ranks",
               "h2d_bytes_per_run": rec.h2d, "d2h_bytes_per_run": rec.d2h}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        del sim
        cpu = cpu_baseline(args, sc)

    # the batched and adjoint ratios, each on its own workload with its own clock record (one GPU)
    extras = {}
    if world == 1 and not args.no_extras:
        bat = run_batched(argparse.Namespace(steps=1500, count=192))
        extras["batched_speedup"] = {
            "value": bat["value"], "unit": "x", "workload": bat["config"]["workload"], "steps": bat["steps"],
            "batched_ms": bat["batched_ms"], "sequential_ms": bat["sequential_ms"], "tuned": bat["tuned"],
            "timing": bat["timing"], "clocks": bat["clocks"]}
        adj = run_adjoint(argparse.Namespace(steps=4000, warmup=3, checkpoints=64, fd=0))
        extras["adjoint_grad_over_forward"] = {
            "value": adj["value"], "unit": "x", "higher_is_better": False, "workload": adj["config"]["workload"],
            "steps": adj["steps"], "checkpoints": adj["config"]["checkpoints"], "forward_ms": adj["forward_ms"],
            "gradient_ms": adj["gradient_ms"], "parts_ms": adj["gradient_parts_ms"],
            "timing": "device time of the forward and of the gradient (forward with checkpoints + recomputation + "
                      "backward sweep), medians of 3 after 3 warm-ups", "clocks": adj["clocks"]}

    if rank == 0:
        line = {
            "metric": "Mcell-updates/s", "value": value, "unit": "Mcell/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": sc.name, "nodes": nn, "cells": sc.grid.cells(), "pml": sc.info.get("pml"),
                       "spheres": sc.info.get("spheres"), "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (6.5 GB of fields per buffer set)",
                       "variant": variant, "coef_classes": classes, "debye_edges": debye_edges,
                       "launches_per_step": launches, "setup_s": round(t_setup, 2)},
            "hbm_fraction_of_algorithmic": BYTES_PER_NODE * value * 1e6 / world / 1e9 / peak,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic_for(dom_name, sc.name), "kernel": dom_name,
                         "kernels": field_parts,
                         "bytes_per_launch": BYTES_PER_NODE * nn, "kernel_ms": dom_ms, "peak_source": peak_src},
            "kernel_ms": {k: round(v, 5) for k, v in kt.items()},
            "kernel_share": {k: round(v / total_kt, 4) for k, v in kt.items()},
            "gpu_launches": launches * K,
            "clocks": clocks,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "energy_after": energy,
            **extras,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
