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


def profile_traffic(precision="f64"):
    """DRAM bytes per fused-step launch from the committed ncu summary of the
    fluid kernel of this storage precision (the FP64 two-cell kernel, or the
    16-bit word kernel), if any."""
    name = {"f64": "lbib_fluid_step_c1.md", "f16": "lbib_fluid_step_words_f16_c1.md"}.get(precision.split("-")[0])
    if name is None:
        return None
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_launch_full:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def gpu_local(make):
    """Run make() with this process bound to the host cores NVML reports as
    local to the current GPU, then restore the binding.  Page-locked buffers
    allocated there sit in the GPU's own NUMA node, so device-to-host copies
    into them do not cross the socket link (a remote node measured up to 5x
    slower).  Without NVML, make() runs unbound."""
    try:
        import pynvml
        import torch
        pynvml.nvmlInit()
        bus = torch.cuda.get_device_properties(torch.cuda.current_device())
        bid = f"{bus.pci_domain_id:08x}:{bus.pci_bus_id:02x}:{bus.pci_device_id:02x}.0"
        h = pynvml.nvmlDeviceGetHandleByPciBusId_v2(bid.encode())
        words = pynvml.nvmlDeviceGetCpuAffinity(h, (os.cpu_count() + 63) // 64)
        local = {64 * w + b for w, m in enumerate(words) for b in range(64) if (m >> b) & 1}
        old = os.sched_getaffinity(0)
        local &= old
        if not local:
            return make()
        os.sched_setaffinity(0, local)
        try:
            return make()
        finally:
            os.sched_setaffinity(0, old)
    except Exception:
        return make()


# ---------------------------------------------------------------- clocks
class Clocks:
    """SM clocks and clock-event reasons sampled DURING a timed region.

    NVML (nvidia-ml-py) from a background thread every `period_s` (5 ms), so
    that even a region of a few tens of milliseconds gets several samples;
    the device is found by its PCI bus id (CUDA and NVML number devices
    differently under CUDA_VISIBLE_DEVICES).  Falls back to `nvidia-smi
    -lms 200` where NVML cannot be used.  Only reads: no setting of the GPU
    is changed."""

    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("sw_power_cap", 0x4))

    def __init__(self, index, period_s=0.005):
        self.index = index
        self.period = period_s
        self.rows = []
        self._thread = None
        self._stop = None
        self._smi = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId_v2(bus.encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        import threading
        self.rows = []
        try:
            nv, h = self._handle()
        except Exception:
            return self._start_smi()
        smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        self._stop = threading.Event()

        def loop():
            while True:
                try:
                    sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                    rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                    self.rows.append((sm, smax, rs))
                except Exception:
                    pass
                if self._stop.wait(self.period):
                    break
        self._thread = threading.Thread(target=loop, daemon=True)
        self._thread.start()

    def _start_smi(self):
        fd, self._path = tempfile.mkstemp(prefix="lbib_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self._smi = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,"
                                          "clocks_event_reasons.active", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self._path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self._smi = None

    def stop(self):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
            self._thread = None
            how = "nvml"
        elif self._smi is not None:
            self._smi.send_signal(signal.SIGTERM)
            try:
                self._smi.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._smi.kill()
            self._smi = None
            for line in open(self._path):
                parts = [p.strip() for p in line.split(",")]
                try:
                    self.rows.append((float(parts[0]), float(parts[1]), int(parts[2], 16)))
                except (ValueError, IndexError):
                    continue
            os.unlink(self._path)
            how = "nvidia-smi"
        else:
            return None
        if not self.rows:
            return None
        reasons = sorted({name for _, _, rs in self.rows for name, bit in self.REASONS if rs & bit})
        return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": max(r[1] for r in self.rows),
                "sm_mhz_min": min(r[0] for r in self.rows), "reasons": reasons, "samples": len(self.rows),
                "sampler": how}


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
    cfg = config_block(args)
    cfg["measured_on"] = ("a bounded sample of the workload: " + sample + "; MLUPS of the reference's CPU step "
                          "are per lattice site, so a sample with the same cross-section, sheet and physics "
                          "stands for the full channel")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": 1, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg,
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
    e0.record(stream)
    solver.run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = solver.kernel_launches - launches0
    ms = e0.elapsed_time(e1)
    group.barrier()
    ms_max = group.max(ms)
    value = whole_job_mlups(case.ncells, args.steps, world, ms_max / 1e3)
    # stage times for the roofline: the same number of steps again, after the
    # timed region, with an event pair around every stage (the events cost
    # tens of microseconds per step, so they stay out of `value`)
    stage_ms, nprof = profiled_steps(solver, args.steps)

    fluid_cells = (case.nx - 4) * (case.ny - 4) * (case.nz - 4)
    bytes_launch = fluid_cells * 19 * 2 * pop_bytes(args.precision)
    fluid_ms = stage_ms["fluid"] / max(nprof, 1)
    achieved = bytes_launch / (fluid_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profile_traffic(args.precision)

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
        # page-locked host memory (a copy to pageable memory is staged by the
        # driver at a fraction of the link speed); made and touched before the
        # timed region, as a caller sets up its output buffers once
        fields = gpu_local(lambda: [torch.empty(case.ncells, dtype=torch.float64, pin_memory=True).numpy()
                                    for _ in range(4)])
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
        t_f = time.perf_counter()
        rho, ux, uy, uz = solver.moments(out=fields)           # D2H: final rho, u fields
        t1 = time.perf_counter()
        e2e_s = group.max(t1 - t0)
        steps_s = group.max(t_f - t0)
        h2d = S * 96
        d2h = S * 96 + 4 * 8 * case.ncells / args.steps
        e2e = {"value": whole_job_mlups(case.ncells, args.steps, world, e2e_s), "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h,
               "how": "lbib_set_sheet + init_df1/init_df_inout, then per step do_thread(1 step) + "
                      "lbib_sync_to_host (sheet records to the host), then lbib_get_moments into the caller's "
                      "page-locked host arrays; wall clock, max over ranks",
               "breakdown": {"steps_ms": steps_s * 1e3, "final_fields_ms": (e2e_s - steps_s) * 1e3,
                             "final_fields_bytes": 4 * 8 * case.ncells,
                             "value_without_final_fields": whole_job_mlups(case.ncells, args.steps, world, steps_s),
                             "note": "the one-off rho/u read-back (4 FP64 fields) amortises over a run's steps: "
                                     f"here {args.steps} steps"}}

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
    c2_leg = None
    if args.c2_steps > 0 and args.precision == "f64":
        c2_leg = run_c2_leg(args, group, peak)
    sur_leg = None
    if args.sur_train > 0 and args.precision == "f64" and world == 1:
        sur_leg = run_surrogate_leg(args)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "f64" else f"{args.precision} storage, f32 arithmetic",
                "data": "synthetic",
                "config": config_block(args),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                             "kernel": ("lbib_fluid_step (fused D3Q19 AA step)" if args.precision == "f64" else
                                        "lbib_fluid_step_words (fused D3Q19 AA step, 16-bit words)"),
                             "bytes_per_launch": bytes_launch, "launch_ms": fluid_ms},
                "stages_ms_per_step": {k: v / max(nprof, 1) for k, v in stage_ms.items()},
                "gpu_launches": launches, "autotune": tuned, "fp16_store": lp,
                "e2e": e2e, "cpu_baseline": cpu, "clocks": clk, "sweep": sweep_leg, "c2": c2_leg,
                "surrogate": sur_leg}
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
        ncomp = int(np.sum(r["completed"]))
        out[prec] = {"points_per_s": group.world * len(probs) / wall, "wall_s": wall,
                     "completed_points": ncomp, "completed_points_per_s": group.world * ncomp / wall,
                     "site_steps_executed": r["site_steps"],
                     "executed_mlups": group.world * r["site_steps"] / wall / 1e6,
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
            "note": "a point whose sheet left its grid stops there and counts as run in points_per_s; "
                    "completed_points_per_s counts only the points that reached the last step, and "
                    "executed_mlups the lattice-site steps actually advanced (a stopped point's sites up to its "
                    "stop step) over the wall time; tips are compared on the points both runs completed"}


def run_c2_leg(args, group, peak):
    """The 512^3 precision workload: tau 0.55, inflow u_x 0.02, two 256 x 256
    sheets (spacing 0.5) at x = 128 and x = 320, Ks and Kb drawn log-uniform
    by numpy default_rng(0) (precision.sweep_case("c2")).  FP64 storage (the
    drop-in), FP16 deviations from the inflow equilibrium ("f16-flow") and
    FP16 deviations from the rest weights ("f16", the f - w shift) each run
    the same `c2_steps` steps from the same initial state, device-timed; the
    last 100 steps are also timed per stage for the fluid kernels' roofline.
    Errors of the FP16 forms against the FP64 state: velocity relative L2
    over the interior, mass against FP64 and each run's own mass drift,
    sheet-tip displacement.  The span is the physical one: under the
    reference's explicit IB coupling this workload's FP64 run stays near
    max|u| ~ 1.3 u_l until ~2250 steps, then diverges and a stencil leaves
    the grid near step 3000, so its 5000 steps cannot be run by FP64."""
    import precision
    case = precision.sweep_case("c2")
    steps = args.c2_steps
    cells = case.nx * case.ny * case.nz
    fluid_cells = (case.nx - 4) * (case.ny - 4) * (case.nz - 4)
    out = {"workload": f"c2: {case.nx}x{case.ny}x{case.nz} D3Q19, tau {case.tau}, u {case.u_l}, two 256x256 sheets "
                       f"at x=128, 320, Ks {case.Ks_l:.4g}, Kb {case.Kb_l:.4g} (default_rng(0)), {steps} steps",
           "steps": steps, "span_note": "FP64 itself diverges after ~2250 steps on this workload (explicit IB "
                                        "coupling), so the comparison runs over the physical span, not 5000 steps"}
    group.barrier()
    ref = precision.run_case(case, steps, "f64", profile_steps=100)
    v64 = cells * steps / ref.seconds / 1e6

    def leg(r, prec):
        fl = r.stages_ms.get("fluid", 0.0)
        b = fluid_cells * 19 * 2 * pop_bytes(prec)
        return {"mlups": cells * steps / r.seconds / 1e6, "ms_per_step": r.seconds * 1e3 / steps,
                "roofline": {"bound": "hbm", "achieved": b / (fl / 1e3) / 1e9 if fl else None, "peak": peak,
                             "unit": "GB/s", "frac": b / (fl / 1e3) / 1e9 / peak if fl else None,
                             "bytes_per_launch": b, "launch_ms": fl},
                "stages_ms_per_step": r.stages_ms}
    out["f64"] = leg(ref, "f64")
    out["f64"]["mass_drift"] = ref.mass / ref.mass0 - 1.0
    for key, prec in (("f16_flow", "f16-flow"), ("f16_fw", "f16")):
        group.barrier()
        r = precision.run_case(case, steps, prec, autotune=True, profile_steps=100)
        d = leg(r, prec)
        d["form"] = prec + (" (deviations from the inflow equilibrium)" if prec.endswith("flow")
                            else " (deviations from the rest weights, f - w)")
        d["variant"] = r.variant
        d["speedup_vs_f64"] = d["mlups"] / v64
        d.update(precision.compare(ref, r, case))
        out[key] = d
        del r
    del ref
    return out


def run_surrogate_leg(args):
    """The learned sweep (surrogate.py): training runs of the batched solver
    (96 x 48 x 48, 32 x 32 free sheet, T = 3000, default_rng(2)), the MLP
    trained by the library's own tcgen05 kernels, re-run thresholds
    calibrated on a quarter of the training runs, then held-out sweep points
    (default_rng(3)) screened -- reported by the surrogate or re-run by the
    batched solver in FP16 storage -- against the plain FP64 batched sweep
    of the same points, which also judges every point (tip displacement of
    the last fiber row within 2%, or 0.02 lattice units).  Sizes are cut
    from the workload's 4096 / 2048 so that the leg stays near two minutes;
    the line states them."""
    import surrogate
    t0 = time.perf_counter()
    r = surrogate.pipeline(train_n=args.sur_train, eval_n=args.sur_eval, steps=3000, every=100,
                           iters=args.sur_iters, members=5, calib_frac=0.25, target=0.99)
    e = r["evaluation"]
    return {"workload": f"learned sweep, 96x48x48 lattice, 32x32 sheet, T=3000: {args.sur_train} training runs "
                        f"(cut from 4096), {args.sur_eval} held-out points (cut from 2048), MLP 5->4x256->192 x5 "
                        f"members, {args.sur_iters} Adam steps of 1024",
            "unit": "points/s",
            "plain_fp64_points_per_s": e["plain_points_per_s"], "plain_fp64_s": e["plain_fp64_s"],
            "surrogate_points_per_s": e["surrogate_points_per_s"], "surrogate_s": e["surrogate_s"],
            "screen_s": e["screen_s"], "rerun_s": e["rerun_s"],
            "speedup_vs_plain_fp64": e["speedup"],
            "reported_by_surrogate": e["reported_by_surrogate"], "rerun": e["rerun"], "rerun_why": e["rerun_why"],
            "rerun_precision": e["rerun_precision"],
            "right_frac": e["right_frac"],
            "right_points_per_s": e["right"] / e["surrogate_s"],
            "reported_completed": e["reported_completed"],
            "reported_completed_tip_within_2pct": e["reported_completed_tip_within_2pct"],
            "completed": e["completed"], "completed_tip_within_2pct": e["completed_tip_within_2pct"],
            "stop_prediction_accuracy": e["stop_prediction_accuracy"],
            "training_runs_s": r["training_runs"]["seconds"], "training_s": r["training"]["seconds"],
            "calibration": r["calibration"], "leg_wall_s": time.perf_counter() - t0,
            "criterion": "a point is right when its stop/complete outcome matches the FP64 run and, if it "
                         "completes, its tip displacement is within 2% (or 0.02 lattice units) of the FP64 run's"}


def profiled_steps(solver, steps):
    """Stage times (ms summed per stage, steps): `steps` more steps with the
    library's per-stage event pairs, outside any timed region."""
    import torch
    solver.profile_begin()
    solver.run(steps)
    stage_ms, nprof = solver.profile_end()
    torch.cuda.synchronize()
    return stage_ms, nprof


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
    e0.record(stream)
    s.run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = group.max(e0.elapsed_time(e1))
    stage_ms, nprof = profiled_steps(s, args.steps)
    world = group.world
    v = whole_job_mlups(case.ncells, args.steps, world, ms / 1e3)
    fluid_cells = (case.nx - 4) * (case.ny - 4) * (case.nz - 4)
    pop = pop_bytes(args.lp_form)
    fluid_ms = stage_ms["fluid"] / max(nprof, 1)
    achieved = fluid_cells * 19 * 2 * pop / (fluid_ms / 1e3) / 1e9
    # error against the FP64 leg, which has run the same warmup + timed +
    # profiled steps
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
                         "launch_ms": fluid_ms, "traffic": profile_traffic(args.lp_form),
                         "kernel": "lbib_fluid_step_words (fused D3Q19 AA step, 16-bit words)"},
            "stages_ms_per_step": {k: x / max(nprof, 1) for k, x in stage_ms.items()},
            "autotune": {"variant": best, "ms_per_step": ms_v},
            "error_vs_f64": {"steps": args.warmup + 2 * args.steps, "velocity_rel_l2": vel,
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
    ap.add_argument("--c2-steps", type=int, default=2000,
                    help="steps of the 512^3 precision leg (FP64 vs FP16 storage; 0: skip)")
    ap.add_argument("--sur-train", type=int, default=2048,
                    help="training runs of the learned-sweep leg (0: skip; one GPU only)")
    ap.add_argument("--sur-eval", type=int, default=512, help="held-out points of the learned-sweep leg")
    ap.add_argument("--sur-iters", type=int, default=8000, help="Adam steps per surrogate member")
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
