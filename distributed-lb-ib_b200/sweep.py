"""Parameter sweeps: many independent LBM-IB problems advanced as one batch.

The sweep workload (the batched-instances benchmark): n problems drawn from
numpy ``default_rng(seed)``, per problem in this order
  nx from {48, 64, 96, 128, 192}, ny and nz each from {32, 48, 64},
  sheet side from 8 to 40 nodes (uniform integer; spacing 0.5),
  Ks log-uniform in [1e-3, 1e-1], Kb log-uniform in [1e-4, 1e-2],
  tau uniform in [0.55, 0.9], inflow u_x uniform in [0.005, 0.03];
the square sheet lies in the plane x = nx/6, centred in y and z, with its
leading row pinned (a flap hinged at its upstream edge; the reference's
sheets are free and drift out of the short channels within the run).

A sweep point is one problem run to the end (or stopped by its own sheet
leaving the grid); points/s = problems / wall-clock seconds of the run.
Each point reports the tip displacement: the mean x-displacement of the
sheet's last fiber row.
"""
from __future__ import annotations

import time
from typing import Dict, List

import numpy as np

import lbib

SIZES_X = (48, 64, 96, 128, 192)
SIZES_YZ = (32, 48, 64)


def make_problem(nx, ny, nz, side, ks, kb, tau, u, pinned=True) -> lbib.Problem:
    w = 0.5 * (side - 1)
    return lbib.Problem(nx, ny, nz, tau, u, ks, kb, side, side, w, w, nx / 6.0,
                        (ny - 1) / 2.0 - w / 2.0, (nz - 1) / 2.0 - w / 2.0, int(pinned))


def draw_problems(n: int = 256, seed: int = 1, pinned: bool = True) -> List[lbib.Problem]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = int(rng.choice(SIZES_X))
        ny = int(rng.choice(SIZES_YZ))
        nz = int(rng.choice(SIZES_YZ))
        side = int(rng.integers(8, 41))
        ks = float(10 ** rng.uniform(-3, -1))
        kb = float(10 ** rng.uniform(-4, -2))
        tau = float(rng.uniform(0.55, 0.9))
        u = float(rng.uniform(0.005, 0.03))
        out.append(make_problem(nx, ny, nz, side, ks, kb, tau, u, pinned))
    return out


def tip_displacement(sheet0: np.ndarray, sheet: np.ndarray) -> float:
    return float(np.mean(sheet[-1, :, 0] - sheet0[-1, :, 0]))


def run_sweep(problems, steps: int, precision: str = "f16-flow", autotune: bool = True,
              compat: int = 0) -> Dict:
    """Advance all problems `steps` steps as one batch: wall-clock and device
    time, per-problem status and tip displacement.  compat 0: the corrected
    boundary loops (the reference's loop-bound slips are a parity matter)."""
    import torch

    t_setup = time.perf_counter()
    b = lbib.Batch(problems, precision, compat=compat)
    try:
        tuned = None
        if autotune and b.variants() > 1:
            _, ms = b.autotune(6)
            tuned = {"classes": int(ms.shape[0]), "best_variant_per_class": [int(i) for i in ms.argmin(axis=1)]}
        sheets0 = [b.sheet(k) for k in range(len(b))]
        b.synchronize()
        t_setup = time.perf_counter() - t_setup
        stream = torch.cuda.ExternalStream(b.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = b.kernel_launches
        t0 = time.perf_counter()
        e0.record(stream)
        b.run(steps)
        e1.record(stream)
        e1.synchronize()
        wall = time.perf_counter() - t0
        gpu_s = e0.elapsed_time(e1) / 1e3
        codes, failed_at = b.status()
        tips = [tip_displacement(sheets0[k], b.sheet(k)) for k in range(len(b))]
        # lattice-site steps advanced: a stopped problem's sites up to its stop step
        ran = np.where(codes != 0, np.minimum(failed_at, steps), steps)
        site_steps = int(sum(p.nx * p.ny * p.nz * int(n) for p, n in zip(problems, ran)))
        cells = b.cells
        launches = b.kernel_launches - l0
    finally:
        b.close()
    return {"precision": precision, "problems": len(problems), "steps": steps,
            "points_per_s": len(problems) / wall, "wall_s": wall, "gpu_s": gpu_s, "setup_s": t_setup,
            "mlups": cells * steps / gpu_s / 1e6, "cells": cells, "kernel_launches": launches,
            "stopped": int((codes != 0).sum()), "stopped_at": [int(s) for s in failed_at[codes != 0]],
            "completed": [bool(c == 0) for c in codes], "site_steps": site_steps,
            "tip_displacement": tips, "autotune": tuned}


def main(argv=None) -> int:
    import argparse
    import json

    ap = argparse.ArgumentParser(description="batched parameter sweep")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--precision", default="f16-flow")
    ap.add_argument("--free", action="store_true", help="sheets not pinned (the reference's free sheets)")
    ap.add_argument("--no-autotune", action="store_true", help="default kernel variant for every size class")
    a = ap.parse_args(argv)
    rep = run_sweep(draw_problems(a.n, a.seed, not a.free), a.steps, a.precision, autotune=not a.no_autotune)
    print(json.dumps(rep))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
