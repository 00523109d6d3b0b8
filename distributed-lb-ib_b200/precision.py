"""Error of the low-precision population storage against the FP64 drop-in.

Runs the same case twice on the GPU -- FP64 storage (the drop-in, equal to
the reference to rounding) and FP32 / FP16 / BF16 storage with FP32
arithmetic -- and states three errors of the low-precision run:

* velocity: relative L2 of u as a vector field over the fluid interior,
  ||u - u64|| / ||u64||;
* mass drift: (M - M64) / M64 with M the FP64 sum of all populations of the
  interior (lbib_conservation_sums), and each run's own drift M(T)/M(0) - 1;
* sheet tip: the tip displacement d = mean x-displacement X(T) - X(0) of
  the sheet's last fiber row (row = rows - 1), against the FP64 run's,
  |d - d64| / |d64| (the worst sheet), and the largest node-position
  difference over all nodes relative to the largest FP64 displacement.

MLUPS count every lattice site, nx*ny*nz, per step.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Dict, List

import numpy as np

import lbib


def tip_displacement(sheet0: np.ndarray, sheet: np.ndarray) -> float:
    """Mean x-displacement of the last fiber row ([rows, cols, 12] records)."""
    return float(np.mean(sheet[-1, :, 0] - sheet0[-1, :, 0]))


@dataclass
class RunState:
    precision: str
    steps: int
    seconds: float
    u: np.ndarray               # [3, nz-4, ny-4, nx-4]
    rho: np.ndarray
    mass0: float
    mass: float
    sheets0: List[np.ndarray] = field(default_factory=list)
    sheets: List[np.ndarray] = field(default_factory=list)


def run_case(case, steps: int, precision: str, chunk: int = 500) -> RunState:
    """Advance `case` for `steps` steps in `precision`; device-timed seconds."""
    import torch

    s = lbib.Solver(case, precision=precision)
    try:
        sheets0 = [s.sheet(k) for k in range(len(case.sheets))]
        mass0 = float(s.conservation()[0])
        stream = torch.cuda.ExternalStream(s.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        left = steps
        while left > 0:
            n = min(chunk, left)
            s.run(n)
            left -= n
        e1.record(stream)
        e1.synchronize()
        rho, ux, uy, uz = s.moments()
        sl = (slice(2, case.nz - 2), slice(2, case.ny - 2), slice(2, case.nx - 2))
        return RunState(precision, steps, e0.elapsed_time(e1) / 1e3,
                        np.stack([ux[sl], uy[sl], uz[sl]]), rho[sl].copy(), mass0,
                        float(s.conservation()[0]), sheets0,
                        [s.sheet(k) for k in range(len(case.sheets))])
    finally:
        s.close()


def compare(ref: RunState, lp: RunState, case) -> Dict[str, float]:
    du = lp.u - ref.u
    out = {
        "velocity_rel_l2": float(np.linalg.norm(du) / max(np.linalg.norm(ref.u), 1e-300)),
        "rho_rel_l2": float(np.linalg.norm(lp.rho - ref.rho) / np.linalg.norm(ref.rho)),
        "mass_vs_f64": (lp.mass - ref.mass) / ref.mass,
        "mass_drift": lp.mass / lp.mass0 - 1.0,
        "mass_drift_f64": ref.mass / ref.mass0 - 1.0,
    }
    tip, nodes = 0.0, 0.0
    for k, sh in enumerate(case.sheets):
        d64 = tip_displacement(ref.sheets0[k], ref.sheets[k])
        dlp = tip_displacement(lp.sheets0[k], lp.sheets[k])
        tip = max(tip, abs(dlp - d64) / max(abs(d64), 1e-300))
        dmax = np.max(np.linalg.norm(ref.sheets[k][..., :3] - ref.sheets0[k][..., :3], axis=-1))
        dnode = np.max(np.linalg.norm(lp.sheets[k][..., :3] - ref.sheets[k][..., :3], axis=-1))
        nodes = max(nodes, float(dnode / max(dmax, 1e-300)))
    out["tip_displacement_rel"] = tip
    out["node_position_rel"] = nodes
    return out


def error_report(case, steps: int, precisions=("f32", "f16", "bf16", "f16-flow", "bf16-flow")) -> Dict[str, Dict[str, float]]:
    """Errors of each low-precision run against the FP64 run, plus timings."""
    t0 = time.time()
    ref = run_case(case, steps, "f64")
    cells = case.nx * case.ny * case.nz
    rep = {"f64": {"seconds": ref.seconds, "mlups": cells * steps / ref.seconds / 1e6,
                   "mass_drift": ref.mass / ref.mass0 - 1.0}}
    for p in precisions:
        try:
            lp = run_case(case, steps, p)
        except lbib.LbibError as e:  # e.g. a sheet driven off the grid by a diverged run
            rep[p] = {"failed": str(e)}
            continue
        r = compare(ref, lp, case)
        r["seconds"] = lp.seconds
        r["mlups"] = cells * steps / lp.seconds / 1e6
        rep[p] = r
    rep["wall_seconds"] = time.time() - t0
    return rep
