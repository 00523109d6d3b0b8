#!/usr/bin/env python
"""Throughput of the FP64 LBM-IB time step on B200, in MLUPS.

Workload (default ``--config c1``): D3Q19 BGK + Guo forcing on a
512(x) x 256 x 256 lattice, tau = 0.6, inflow u_x = 0.01, one 208 x 208
fiber sheet (spacing 0.5) at x = 80 with Ks = 0.05, Kb = 0.005 -- the
drop-in path, FP64, bit-faithful to the reference's arithmetic.  A step is
one full LBM-IB step (fiber forces, spread, fused fluid step, moments on the
touched tiles, interpolate + move).  Inputs (populations, 5.1 GB) are far
larger than L2, so no flush is needed between steps.

Line fields: ``value`` = lattice updates per second over all ranks with the
state resident in HBM (CUDA events on the library's stream, max over ranks);
``e2e`` = the same through the reference-facing C ABI with host buffers: the
sheet uploaded from host memory and the initial state built, then every
step followed by a device->host read of the sheet records, and the final
rho/u fields read back -- all inside the timed region; ``roofline`` = the
fused fluid kernel's algorithmic bytes per launch over its event-timed
duration, against the measured HBM copy bandwidth; ``cpu_baseline`` = the
reference's own pthread code (oracle/_ref) on a bounded sample, rank 0.

``--impl reference`` times the reference's CPU implementation (oracle/_ref,
all host threads it can use) on a bounded sample of the same workload.
Multi-GPU (``--gpus N`` under torchrun): N independent replicas, one per GPU
(weak scaling); the step has no exchange, so there is no collective.
"""
from __future__ import annotations

import argparse
import json
import os
import signal
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "distributed-lb-ib_b200")
sys.path.insert(0, PKG)

METRIC = "MLUPS & % HBM roofline, FP64 vs FP16-store; sweep pts/s at ≤2% tip error"
UNIT = "MLUPS"
BYTES_PER_UPDATE = 19 * 8 * 2  # FP64 populations read once + written once


class Sheet:
    def __init__(self, rows, cols, width, height, x0, y0, z0):
        self.rows, self.cols, self.width, self.height = rows, cols, width, height
        self.x0, self.y0, self.z0 = x0, y0, z0


class Case:
    def __init__(self, nx, ny, nz, sheets, tau=0.6, u_l=0.01, Ks_l=0.05, Kb_l=0.005, cube_size=4, compat=7):
        self.nx, self.ny, self.nz, self.sheets = nx, ny, nz, sheets
        self.tau, self.u_l, self.Ks_l, self.Kb_l = tau, u_l, Ks_l, Kb_l
        self.cube_size, self.compat = cube_size, compat

    @property
    def ncells(self):
        return self.nx * self.ny * self.nz


def centred(nx, ny, nz, rows, cols, spacing, x0):
    w, h = spacing * (cols - 1), spacing * (rows - 1)
    return Sheet(rows, cols, w, h, x0, (ny - 1) / 2.0 - h / 2.0, (nz - 1) / 2.0 - w / 2.0)


CONFIGS = {
    # the headline configuration: 512 x 256 x 256, 208 x 208 sheet at x = 80
    "c1": dict(nx=512, ny=256, nz=256, rows=208, cols=208, x0=80.0),
    # the reference's own size: 128 x 64 x 64, 52 x 52 sheet at x = 20
    "c0": dict(nx=128, ny=64, nz=64, rows=52, cols=52, x0=20.0),
    # c1 at half size per axis (populations 637 MB, above L2): for ncu captures
    "p1": dict(nx=256, ny=128, nz=128, rows=104, cols=104, x0=40.0),
}


def make_case(name):
    c = CONFIGS[name]
    return Case(c["nx"], c["ny"], c["nz"], [centred(c["nx"], c["ny"], c["nz"], c["rows"], c["cols"], 0.5, c["x0"])])


def cpu_sample_case(name):
    """A bounded CPU sample of the workload: the same y-z cross-section, sheet
    and physics, with the channel shortened to 128 cells (c1) so that the
    reference's 824-byte-per-cell layout and step time stay bounded."""
    c = dict(CONFIGS[name])
    if c["nx"] > 128:
        c["nx"] = 128
    return Case(c["nx"], c["ny"], c["nz"], [centred(c["nx"], c["ny"], c["nz"], c["rows"], c["cols"], 0.5, c["x0"])])


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per fused-step launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "lbib_fluid_step_c1.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_launch_full:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi samples during the timed region (own PID, stopped after)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="lbib_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smax=float(parts[2]), power=float(parts[3]),
                                 hw=parts[5], hwt=parts[6], swt=parts[7], swp=parts[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        reasons = set()
        for r in rows:
            for k, name in [("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                            ("swt", "sw_thermal_slowdown"), ("swp", "sw_power_cap")]:
                if r[k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in rows), "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------- ranks
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Group:
    """torch.distributed for the barrier and the max over ranks: NCCL, one
    rank per GPU, on a GPU box; gloo when there is no GPU (host-side tests)."""

    def __init__(self, world, local, backend=None, timeout_s=300):
        self.world = world
        self.dist = None
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            kw = {}
            if self.backend == "nccl":
                torch.cuda.set_device(local)
                kw["device_id"] = torch.device("cuda", local)
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist
            self.torch = torch

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, v):
        if not self.dist:
            return v
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = self.torch.tensor([v], dtype=self.torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()


def whole_job_mlups(cells_per_rank, steps, world, max_seconds):
    """Lattice updates of all replicas over the slowest rank's time."""
    return cells_per_rank * steps * world / max_seconds / 1e6


# ---------------------------------------------------------------- CPU legs
def cpu_reference_time(name, steps, threads=None):
    """Seconds per step of the reference's pthread code on a bounded sample
    (oracle/_ref, P = 1, Q x R threads); falls back to the oracle port."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as P
    case = cpu_sample_case(name)
    oc = P.Case(case.nx, case.ny, case.nz,
                [P.Sheet(s.rows, s.cols, s.width, s.height, s.x0, s.y0, s.z0) for s in case.sheets],
                case.tau, case.u_l, case.Ks_l, case.Kb_l)
    cores = threads or os.cpu_count() or 1
    ncy, ncz = case.ny // 4, case.nz // 4
    if not P.reference_available():
        try:
            P.build()
        except RuntimeError:
            pass
    if P.reference_available():
        # largest Q*R <= cores with Q | ncy, R | ncz, even total (reference's check)
        best = (1, 1)
        for q in range(1, ncy + 1):
            if ncy % q:
                continue
            for r in range(1, ncz + 1):
                if ncz % r or q * r > cores or (q * r) % 2 or q * r > case.sheets[0].rows:
                    continue
                if q * r > best[0] * best[1]:
                    best = (q, r)
        ref = P.Reference(oc)
        ref.run_threaded(1, *best)            # step 1 writes the reference's FieldView files
        t0 = time.perf_counter()
        ref.run_threaded(steps, *best)
        dt = (time.perf_counter() - t0) / steps
        del ref
        return dt, case, best[0] * best[1], "reference"
    P.Oracle.set_threads(cores)
    o = P.Oracle(oc)
    o.run(1)
    t0 = time.perf_counter()
    o.run(steps)
    dt = (time.perf_counter() - t0) / steps
    return dt, case, cores, "port"


def run_reference(args):
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    steps = max(1, min(args.steps, args.cpu_steps))
    dt, case, cores, kind = cpu_reference_time(args.config, steps)
    v = case.ncells / dt / 1e6
    sample = (f"{case.nx}x{case.ny}x{case.nz} lattice (the {args.config} cross-section, channel cut to "
              f"{case.nx}), {case.sheets[0].rows}x{case.sheets[0].cols} sheet, {steps} steps after 1 untimed")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": 1, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_block(args),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def pop_bytes(precision):
    return {"f64": 8, "f32": 4}.get(precision.split("-")[0], 2)


def config_block(args):
    c = CONFIGS[args.config]
    prec = getattr(args, "precision", "f64")
    store = "FP64" if prec == "f64" else f"{prec} storage / FP32 arithmetic"
    gb = c["nx"] * c["ny"] * c["nz"] * 19 * pop_bytes(prec) / 1e9
    return {"workload": f"{args.config}: {store} LBM-IB step, {c['nx']}x{c['ny']}x{c['nz']} D3Q19 lattice, "
                        f"{c['rows']}x{c['cols']} fiber sheet at x={c['x0']:g}, tau 0.6, u 0.01, Ks 0.05, Kb 0.005",
            "lattice": [c["nx"], c["ny"], c["nz"]], "sheet": [c["rows"], c["cols"]],
            "parallelism": f"replicas x{args.gpus}",
            "l2_flush": f"inputs ({gb:.2f} GB populations) vs 126 MB L2" + (" -- larger, no flush needed"
                                                                              if gb > 0.5 else "")}


# ---------------------------------------------------------------- GPU leg
def run_lbib(args):
    world, rank, local = dist_env()
    import numpy as np

    import lbib
    if not os.path.exists(lbib.LIB_PATH):
        lbib.build()
    group = Group(world, local)
    import torch
    torch.cuda.set_device(local)
    case = make_case(args.config)
    solver = lbib.Solver(case, precision=args.precision)
    tuned = None
    if args.variant is not None:
        solver.set_variant(args.variant)
    elif solver.variants() > 1:
        best, ms_v = solver.autotune(8)
        tuned = {"variant": best, "ms_per_step": ms_v}
    init_sheet = np.ascontiguousarray(solver.sheet(0))   # the host copy a user starts from
    stream = torch.cuda.ExternalStream(solver.stream)
    solver.run(args.warmup)
    solver.synchronize()

    # ---- device-resident throughput (value) and stage timing (roofline)
    group.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    launches0 = solver.kernel_launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    solver.profile_begin()
    e0.record(stream)
    solver.run(args.steps)
    e1.record(stream)
    stage_ms, nprof = solver.profile_end()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = solver.kernel_launches - launches0
    ms = e0.elapsed_time(e1)
    group.barrier()
    ms_max = group.max(ms)
    value = whole_job_mlups(case.ncells, args.steps, world, ms_max / 1e3)

    fluid_cells = (case.nx - 4) * (case.ny - 4) * (case.nz - 4)
    bytes_launch = fluid_cells * 19 * 2 * pop_bytes(args.precision)
    fluid_ms = stage_ms["fluid"] / max(nprof, 1)
    achieved = bytes_launch / (fluid_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profile_traffic()

    # ---- the FP16-store form of the same workload, same step count
    lp = None
    if args.precision == "f64" and args.lp_form != "none":
        lp = run_lp_form(args, case, solver, group, value, peak)

    # ---- end to end through the C ABI with host buffers
    S = sum(s.rows * s.cols for s in case.sheets)
    e2e = None
    if not args.no_e2e:
        import numpy as np
        # the caller's host arrays for the final fields exist before the run
        # (allocated and written once here, outside the timed region, so that
        # the OS has mapped their pages)
        fields = [np.empty(case.ncells) for _ in range(4)]
        for a in fields:
            a.fill(0.0)
        group.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solver.set_sheet(0, init_sheet)                        # H2D: the sheet
        lib = solver.lib
        lib.init_df1(solver.gv)                                # initial state on the device
        lib.init_df_inout(solver.gv)
        for _ in range(args.steps):
            solver.run(1)                                      # do_thread for one step
            lib.lbib_sync_to_host(solver.gv)                   # D2H: sheet records into the GV
        rho, ux, uy, uz = solver.moments(out=fields)           # D2H: final rho, u fields
        t1 = time.perf_counter()
        e2e_s = group.max(t1 - t0)
        h2d = S * 96
        d2h = S * 96 + 4 * 8 * case.ncells / args.steps
        e2e = {"value": whole_job_mlups(case.ncells, args.steps, world, e2e_s), "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h,
               "how": "lbib_set_sheet + init_df1/init_df_inout, then per step do_thread(1 step) + "
                      "lbib_sync_to_host, then lbib_get_moments into the caller's (already mapped) host arrays; "
                      "wall clock, max over ranks"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        dt, sc, cores, kind = cpu_reference_time(args.config, args.cpu_steps)
        cpu = {"value": sc.ncells / dt / 1e6, "unit": UNIT, "cores": cores, "kind": kind,
               "sample": f"{sc.nx}x{sc.ny}x{sc.nz} lattice (the {args.config} cross-section, channel cut to "
                         f"{sc.nx}), {sc.sheets[0].rows}x{sc.sheets[0].cols} sheet, {args.cpu_steps} steps"}

    solver.close()
    sweep_leg = None
    if args.sweep_n > 0 and args.precision == "f64":
        sweep_leg = run_sweep_leg(args, group)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "f64" else f"{args.precision} storage, f32 arithmetic",
                "data": "synthetic",
                "config": config_block(args),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                             "kernel": "lbib_fluid_step (fused D3Q19 AA step)",
                             "bytes_per_launch": bytes_launch, "launch_ms": fluid_ms},
                "stages_ms_per_step": {k: v / max(nprof, 1) for k, v in stage_ms.items()},
                "gpu_launches": launches, "autotune": tuned, "fp16_store": lp,
                "e2e": e2e, "cpu_baseline": cpu, "clocks": clk, "sweep": sweep_leg}
        print(json.dumps(line), flush=True)
    group.close()
    return 0


def run_sweep_leg(args, group):
    """The batched parameter sweep (sweep.py: 256 uneven problems, seed 1,
    2000 steps, pinned flaps), once in FP16 storage and once in FP64, each as
    one batch per GPU.  points/s = problems of all ranks / max wall time;
    a point is within 2% when its FP16 tip displacement is within 2% of its
    FP64 one (both runs reached the end)."""
    import numpy as np

    import sweep
    probs = sweep.draw_problems(args.sweep_n, 1)
    out = {}
    for prec in ("f16-flow", "f64"):
        group.barrier()
        r = sweep.run_sweep(probs, args.sweep_steps, prec)
        wall = group.max(r["wall_s"])
        out[prec] = {"points_per_s": group.world * len(probs) / wall, "wall_s": wall,
                     "mlups": r["mlups"], "gpu_launches": r["kernel_launches"], "stopped": r["stopped"],
                     "autotuned_size_classes": (r["autotune"] or {}).get("classes"),
                     "tips": r["tip_displacement"], "completed": r["completed"]}
    t16, t64 = np.array(out["f16-flow"].pop("tips")), np.array(out["f64"].pop("tips"))
    both = np.array(out["f16-flow"].pop("completed")) & np.array(out["f64"].pop("completed"))
    stopped16 = out["f16-flow"]["stopped"]
    rel = np.abs(t16 - t64) / np.maximum(np.abs(t64), 1e-3)
    ok = both & (rel <= 0.02)
    miss = [{"problem": int(i), "tip_fp64": float(t64[i]), "tip_fp16": float(t16[i])}
            for i in np.nonzero(both & ~ok)[0]]
    return {"workload": f"{len(probs)} problems (sweep.py, seed 1), {args.sweep_steps} steps, one batch per GPU",
            "unit": "points/s", "fp16_batched": out["f16-flow"], "fp64_batched": out["f64"],
            "speedup_fp16_vs_fp64": out["f16-flow"]["points_per_s"] / out["f64"]["points_per_s"],
            "completed_both": int(both.sum()), "tip_within_2pct_of_fp64": int(ok.sum()), "stopped_fp16": stopped16,
            "tip_rel_err_median": float(np.median(rel[both])) if both.any() else None,
            "tip_outside_2pct": miss,
            "note": "a point whose sheet left its grid stops there and counts as run; tips are compared on "
                    "the points both runs completed"}


def run_lp_form(args, case, ref_solver, group, value64, peak):
    """Time the low-precision storage form (default f16-flow: FP16 deviations
    from the inflow equilibrium, FP32 arithmetic) on the same workload and
    step count as the FP64 leg, and state its error against that FP64 state."""
    import numpy as np
    import torch

    import lbib
    import precision
    s = lbib.Solver(case, precision=args.lp_form)
    sheet0 = s.sheet(0)
    best, ms_v = s.autotune(8)
    stream = torch.cuda.ExternalStream(s.stream)
    s.run(args.warmup)
    s.synchronize()
    group.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.profile_begin()
    e0.record(stream)
    s.run(args.steps)
    e1.record(stream)
    stage_ms, nprof = s.profile_end()
    torch.cuda.synchronize()
    ms = group.max(e0.elapsed_time(e1))
    world = group.world
    v = whole_job_mlups(case.ncells, args.steps, world, ms / 1e3)
    fluid_cells = (case.nx - 4) * (case.ny - 4) * (case.nz - 4)
    pop = pop_bytes(args.lp_form)
    fluid_ms = stage_ms["fluid"] / max(nprof, 1)
    achieved = fluid_cells * 19 * 2 * pop / (fluid_ms / 1e3) / 1e9
    # error against the FP64 leg, which has run the same warmup + steps
    u64 = np.stack(ref_solver.moments()[1:])
    ulp = np.stack(s.moments()[1:])
    sl = (slice(None), slice(2, case.nz - 2), slice(2, case.ny - 2), slice(2, case.nx - 2))
    vel = float(np.linalg.norm(ulp[sl] - u64[sl]) / np.linalg.norm(u64[sl]))
    d64 = precision.tip_displacement(sheet0, ref_solver.sheet(0))
    dlp = precision.tip_displacement(sheet0, s.sheet(0))
    s.close()
    return {"form": args.lp_form, "value": v, "unit": UNIT, "ms_per_step": ms / args.steps,
            "speedup_vs_f64": v / value64,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "bytes_per_launch": fluid_cells * 19 * 2 * pop,
                         "launch_ms": fluid_ms},
            "stages_ms_per_step": {k: x / max(nprof, 1) for k, x in stage_ms.items()},
            "autotune": {"variant": best, "ms_per_step": ms_v},
            "error_vs_f64": {"steps": args.warmup + args.steps, "velocity_rel_l2": vel,
                             "tip_displacement_rel": abs(dlp - d64) / max(abs(d64), 1e-300)}}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["lbib", "reference"], default="lbib")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="c1")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--sweep-n", type=int, default=256, help="problems of the batched sweep leg (0: skip)")
    ap.add_argument("--sweep-steps", type=int, default=2000)
    ap.add_argument("--lp-form", default="f16-flow",
                    help="low-precision form timed beside the FP64 leg (or 'none')")
    ap.add_argument("--variant", type=int, default=None,
                    help="fluid-kernel variant (default: autotuned when there are several)")
    ap.add_argument("--precision", default="f64",
                    help="population storage of the timed leg: f64 (the drop-in), f32, f16, bf16, *-flow")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    return run_lbib(args)


if __name__ == "__main__":
    sys.exit(main())
