"""Generates the full-size parity fixtures: the oracle (the CPU restatement of sims-field's CPU
FDTD, oracle/) run at the benchmark configurations' full sizes and step counts, in f32 (the
reference's own arithmetic) and f64 (the FP64 truth run of the same update), reduced to what a GPU
run can be compared with cheaply:

  series32 / series64     the port V/I series, every step
  norms32 / norms64       the L2 norm of each field component over the whole grid (Ex..Hz)
  idx                     seeded node indices, the same for every component
  e32, h32 / e64, h64     the final E and H at those nodes (component-major: [3, len(idx)])
  extra per config        plane-DFT or NTFF samples and norms, far fields (the antenna)

Configs (all seeded; fieldgrid_b200.workloads builds the same scenes the tests and bench use):
  spheres512   512^3 cells (513^3 nodes), 200 spheres, 20 % Debye, 10-cell CPML, one 50-ohm port,
               2000 steps                                        (the throughput configuration)
  patch256     256x256x192 cells, 12-cell CPML, PEC patch on a 2-cell substrate over a ground,
               NTFF box 3 cells inside the CPML at 8, 10, 12 GHz, 6000 steps, far field on the
               5-degree theta/phi grid                            (the antenna configuration)
  flux160      160x160x96 cells, 8-cell CPML, the adjoint workload's forward with its plane DFT
               at 10 GHz, 4000 steps                              (the adjoint configuration)

Usage: python tests/golden/make_fullsize.py NAME [--threads N] [--steps S]   (minutes to hours on
a CPU host; writes tests/golden/NAME.npz). Test infrastructure: it runs the oracle as the checker.
"""
from __future__ import annotations

import argparse
import gc
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SAMPLES = 8192           # nodes sampled per field
SAMPLE_SEED = 20261204


def sample_nodes(nn: int, count: int = SAMPLES, seed: int = SAMPLE_SEED) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(nn, size=min(count, nn), replace=False)).astype(np.int64)


def far_dirs() -> np.ndarray:
    """theta = 0..180 and phi = 0..355 degrees in 5-degree steps (37 x 72 directions)."""
    th = np.deg2rad(np.arange(0, 181, 5, dtype=np.float64))
    ph = np.deg2rad(np.arange(0, 360, 5, dtype=np.float64))
    t, p = np.meshgrid(th, ph, indexing="ij")
    return np.stack([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)], -1).reshape(-1, 3)


def scene_of(name: str):
    from fieldgrid_b200 import workloads as W
    if name == "spheres512":
        return W.spheres(512), None
    if name == "patch256":
        return W.patch_antenna(), 3
    if name == "flux160":
        scene, _spec, _e, _s = W.flux_design()
        return scene(), None
    raise SystemExit(f"unknown configuration {name}")


def run_one(name: str, bits: int, steps: int = 0) -> dict:
    from oracle import oracle as O
    sc, inset = scene_of(name)
    if steps:
        sc.extras.max_steps = steps
    t0 = time.time()
    osim = O.OracleSim(*sc.args(), bits=bits)
    out = {}
    if inset is not None:
        pos, area, gpu_patches = O.patches(osim, inset)
        sc.extras.ntff = gpu_patches
        out["patch_pos"], out["patch_area"] = pos, area
    setup = time.time() - t0
    rec = O.run_cpu(osim, 0, sc.pulse, sc.extras, keep_fields=True)
    run_s = time.time() - t0 - setup
    nn = int(np.prod(sc.grid.dims()))
    idx = sample_nodes(nn)
    out["steps"] = rec.steps
    out["series"] = rec.series.copy()
    fields = {}
    norms = []
    for which in ("e", "h"):
        a = getattr(rec, which).reshape(3, nn)
        norms += [float(np.linalg.norm(a[c])) for c in range(3)]
        fields[which] = a[:, idx].copy()
        setattr(rec, which, None)
        del a
        gc.collect()
    out["norms"] = np.array(norms)
    out["e"], out["h"] = fields["e"], fields["h"]
    if rec.plane.size:
        out["plane_norm"] = float(np.linalg.norm(rec.plane))
        out["plane_idx"] = sample_nodes(rec.plane.size, SAMPLES, SAMPLE_SEED + 1)
        out["plane"] = rec.plane[out["plane_idx"]].copy()
    if rec.ntff.size:
        acc = rec.ntff.astype(np.float32)
        out["ntff_norm"] = float(np.linalg.norm(rec.ntff))
        out["ntff_idx"] = sample_nodes(acc.size, SAMPLES, SAMPLE_SEED + 2)
        out["ntff"] = rec.ntff[out["ntff_idx"]].copy()
        dirs = far_dirs()
        nf = len(sc.extras.freqs)
        far = []
        for k, f in enumerate(sc.extras.freqs):
            fld, _ = O.far_eval(out["patch_pos"], out["patch_area"], acc, nf, k, f, dirs)
            far.append(fld)
        out["far"] = np.stack(far)            # [nf, directions, 3] complex
        out["freqs"] = np.array(sc.extras.freqs)
    del rec
    gc.collect()
    print(f"{name} f{bits}: setup {setup:.1f} s, {out['steps']} steps in {run_s:.1f} s "
          f"({nn * out['steps'] / run_s / 1e6:.1f} Mcell/s on {O.threads()} threads)", flush=True)
    out["run_s"] = run_s
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("name", choices=["spheres512", "patch256", "flux160"])
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--steps", type=int, default=0, help="override the configuration's step count")
    a = ap.parse_args()
    if a.threads:
        os.environ["OMP_NUM_THREADS"] = str(a.threads)
    r32 = run_one(a.name, 32, a.steps)
    r64 = run_one(a.name, 64, a.steps)
    sc, _ = scene_of(a.name)
    nn = int(np.prod(sc.grid.dims()))
    save = dict(name=a.name, dims=np.array(sc.grid.dims()), steps=r32["steps"], idx=sample_nodes(nn),
                sample_seed=SAMPLE_SEED, run_s32=r32["run_s"], run_s64=r64["run_s"])
    for key in ("series", "norms", "e", "h", "plane", "plane_idx", "plane_norm", "ntff", "ntff_idx",
                "ntff_norm", "far"):
        if key in r32:
            if key.endswith("_idx"):
                save[key] = r32[key]
                continue
            save[key + "32"] = np.asarray(r32[key], np.float32) if key in ("e", "h") else r32[key]
            save[key + "64"] = r64[key]
    if "freqs" in r32:
        save["freqs"] = r32["freqs"]
    path = os.path.join(HERE, f"{a.name}.npz")
    np.savez_compressed(path, **save)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)")


if __name__ == "__main__":
    main()
