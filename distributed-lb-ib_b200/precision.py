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
    stages_ms: Dict[str, float] = field(default_factory=dict)   # per step, over the profiled steps
    variant: int = -1                                            # autotuned word-kernel variant


def run_case(case, steps: int, precision: str, chunk: int = 500, autotune: bool = False,
             profile_steps: int = 0) -> RunState:
    """Advance `case` for `steps` steps in `precision`; device-timed seconds.
    With `autotune` the fastest fluid-kernel variant is chosen first (the run
    itself is unchanged by it); the last `profile_steps` steps are also timed
    per stage (CUDA events between the stages)."""
    import torch

    s = lbib.Solver(case, precision=precision)
    try:
        variant = -1
        if autotune and s.variants() > 1:
            variant, _ = s.autotune(8)
        sheets0 = [s.sheet(k) for k in range(len(case.sheets))]
        mass0 = float(s.conservation()[0])
        stream = torch.cuda.ExternalStream(s.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        prof = min(max(profile_steps, 0), steps)
        left = steps - prof
        while left > 0:
            n = min(chunk, left)
            s.run(n)
            left -= n
        stages = {}
        if prof:
            s.profile_begin()
            s.run(prof)
            st, n = s.profile_end()
            stages = {k: v / max(n, 1) for k, v in st.items()}
        e1.record(stream)
        e1.synchronize()
        rho, ux, uy, uz = s.moments()
        sl = (slice(2, case.nz - 2), slice(2, case.ny - 2), slice(2, case.nx - 2))
        return RunState(precision, steps, e0.elapsed_time(e1) / 1e3,
                        np.stack([ux[sl], uy[sl], uz[sl]]), rho[sl].copy(), mass0,
                        float(s.conservation()[0]), sheets0,
                        [s.sheet(k) for k in range(len(case.sheets))], stages, variant)
    finally:
        s.close()


def horizon(case, max_steps: int, chunk: int = 250, growth: float = 3.0):
    """How long the FP64 run of `case` stays physical: steps it in chunks,
    recording max |u| after each, until a fiber stencil leaves the grid or
    max_steps.  Returns (trace [(step, max|u|)], failed step or None, the
    last step with max|u| <= growth * u_l)."""
    trace, failed, ok = [], None, 0
    s = lbib.Solver(case, precision="f64")
    try:
        done = 0
        while done < max_steps:
            n = min(chunk, max_steps - done)
            try:
                s.run(n)
            except lbib.LbibError:
                failed = done + n
                break
            done += n
            _, ux, uy, uz = s.moments()
            umax = float(np.sqrt(np.max(ux * ux + uy * uy + uz * uz)))
            del ux, uy, uz
            trace.append((done, umax))
            if umax <= growth * case.u_l and ok == done - n:
                ok = done
    finally:
        s.close()
    return trace, failed, ok


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
    try:
        ref = run_case(case, steps, "f64")
    except lbib.LbibError as e:  # the FP64 run itself left the grid: nothing to compare against
        return {"f64": {"failed": str(e)}, "wall_seconds": time.time() - t0}
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


# ------------------------------------------------------------------ CLI
class _Sheet:
    def __init__(self, rows, cols, width, height, x0, y0, z0):
        self.rows, self.cols, self.width, self.height = rows, cols, width, height
        self.x0, self.y0, self.z0 = x0, y0, z0


class _Case:
    def __init__(self, nx, ny, nz, sheets, tau, u_l, Ks_l, Kb_l, cube_size=4, compat=7):
        self.nx, self.ny, self.nz, self.sheets = nx, ny, nz, sheets
        self.tau, self.u_l, self.Ks_l, self.Kb_l = tau, u_l, Ks_l, Kb_l
        self.cube_size, self.compat = cube_size, compat


def _centred(nx, ny, nz, rows, cols, spacing, x0):
    w, h = spacing * (cols - 1), spacing * (rows - 1)
    return _Sheet(rows, cols, w, h, x0, (ny - 1) / 2.0 - h / 2.0, (nz - 1) / 2.0 - w / 2.0)


def sweep_case(name: str):
    """The precision-sweep workloads.

    c2: 512^3 lattice, tau 0.55, inflow u_x 0.02, two 256x256 sheets
        (spacing 0.5) at x = 128 and x = 320; Ks, Kb drawn log-uniform in
        [1e-3, 1e-1] and [1e-4, 1e-2] by numpy default_rng(0) (one pair,
        shared by both sheets: the solver's Ks, Kb are per problem).
    c0: 128x64x64, one 52x52 sheet at x = 20, tau 0.6, u 0.01, Ks 0.05,
        Kb 0.005 (the reference's own size)."""
    if name == "c2":
        rng = np.random.default_rng(0)
        ks = float(10 ** rng.uniform(-3, -1))
        kb = float(10 ** rng.uniform(-4, -2))
        n = 512
        return _Case(n, n, n, [_centred(n, n, n, 256, 256, 0.5, 128.0), _centred(n, n, n, 256, 256, 0.5, 320.0)],
                     tau=0.55, u_l=0.02, Ks_l=ks, Kb_l=kb)
    if name == "c0":
        return _Case(128, 64, 64, [_centred(128, 64, 64, 52, 52, 0.5, 20.0)], tau=0.6, u_l=0.01, Ks_l=0.05,
                     Kb_l=0.005)
    raise ValueError(name)


def main(argv=None) -> int:
    import argparse
    import json

    ap = argparse.ArgumentParser(description="low-precision storage error against FP64")
    ap.add_argument("--config", default="c2", choices=["c2", "c0"])
    ap.add_argument("--steps", type=int, default=5000,
                    help="steps to compare; with --horizon, the most to try")
    ap.add_argument("--horizon", action="store_true",
                    help="first find how long the FP64 run stays physical and compare over that span")
    ap.add_argument("--forms", default="f32,f16,bf16,f32-flow,f16-flow,bf16-flow")
    a = ap.parse_args(argv)
    case = sweep_case(a.config)
    steps, hz = a.steps, None
    if a.horizon:
        trace, failed, ok = horizon(case, a.steps)
        hz = {"trace_step_umax": trace, "f64_failed_at": failed, "physical_until": ok}
        steps = ok
    rep = error_report(case, steps, tuple(a.forms.split(","))) if steps > 0 else {}
    rep["horizon"] = hz
    rep["config"] = {"name": a.config, "lattice": [case.nx, case.ny, case.nz], "tau": case.tau, "u_l": case.u_l,
                     "Ks_l": case.Ks_l, "Kb_l": case.Kb_l, "steps": steps,
                     "sheets": [[s.rows, s.cols, s.x0] for s in case.sheets]}
    print(json.dumps(rep))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
