"""x-slab decomposition of one LBM-IB grid over several GPUs.

Each slab is a GV holding global columns [x_lo, x_hi) of the grid (bounds
multiples of 4) plus ghost columns, and the whole sheet, whose forces,
spread and move every slab computes alike (the sheet is small next to the
grid).  A step (include/lbib.h, lbib_slab_*):

  1. fluid: forces, spread, fused fluid step on the slab's cells; the face
     columns go into send_lo / send_hi (5 populations x ny x nz each);
  2. exchange the faces: send_lo -> left neighbour's recv_hi, send_hi ->
     right neighbour's recv_lo;
  3. moments: unpack, then the moment tiles of the slab's own columns (-0.0
     in the others);
  4. sum the moment tiles over all slabs (each value has one owner, and
     -0.0 is the identity of the sum, so every slab gets every bit);
  5. move the sheet.

The result is bit-identical to the whole grid on one GPU.  The reference
has no such split (its pthread version shares memory, its MPI version
swaps whole cube faces); the transports here are:

  LocalSlabs   all slabs in one process (one or several GPUs), face copies
               and the tile sum through torch;
  DistSlabs    one slab per rank of a torch.distributed group: NCCL
               send/recv and all-reduce on the slab's CUDA stream, or gloo
               through host memory.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence, Tuple

import numpy as np

import lbib
from lbib import LbibError, _check


def slab_bounds(nx: int, n: int) -> List[Tuple[int, int]]:
    """[x_lo, x_hi) of n slabs over nx columns: multiples of 4, as even as
    they go (the first slabs take the extra tiles)."""
    tiles = nx // 4
    if nx % 4 or n < 1 or n > tiles:
        raise LbibError(f"cannot cut {nx} columns into {n} slabs of whole 4-column tiles")
    q, r = divmod(tiles, n)
    out, lo = [], 0
    for k in range(n):
        hi = lo + 4 * (q + (k < r))
        out.append((lo, hi))
        lo = hi
    return out


def _bind(lib) -> None:
    if getattr(lib, "_slab_bound", False):
        return
    lib.lbib_case_create_slab.restype = C.c_void_p
    lib.lbib_case_create_slab.argtypes = lib.lbib_case_create.argtypes + [C.c_int, C.c_int]
    lib.lbib_set_slab.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.lbib_slab_buffers.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_long)]
    for n in ("lbib_slab_step_fluid", "lbib_slab_step_moments", "lbib_slab_step_move"):
        getattr(lib, n).argtypes = [C.c_void_p]
    lib.lbib_slab_moments.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_long)]
    lib._slab_bound = True


class _Dev:
    """A device array the library owns, seen by torch without a copy."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


def _tensor(ptr: int, n: int):
    import torch
    return torch.as_tensor(_Dev(ptr, n))          # on the device that holds ptr


class SlabSolver(lbib.Solver):
    """One slab [x_lo, x_hi) of `case` (FP64).  The getters return the whole
    grid's shape with this slab's columns filled (see `columns`)."""

    def __init__(self, case, x_lo: int, x_hi: int):
        lib = lbib.load()
        _bind(lib)
        self.lib = lib
        self.case = case
        self.precision = "f64"
        self.x_lo, self.x_hi = x_lo, x_hi
        sh: Sequence = case.sheets
        k = len(sh)
        ia = lambda v: (C.c_int * k)(*v)
        da = lambda v: (C.c_double * k)(*v)
        lib.lbib_clear_error()
        self.gv = lib.lbib_case_create_slab(
            case.nx, case.ny, case.nz, case.cube_size, k,
            ia([s.rows for s in sh]), ia([s.cols for s in sh]),
            da([s.width for s in sh]), da([s.height for s in sh]),
            da([s.x0 for s in sh]), da([s.y0 for s in sh]), da([s.z0 for s in sh]),
            case.tau, case.u_l, case.Ks_l, case.Kb_l, case.compat, x_lo, x_hi)
        if not self.gv:
            rc = lib.lbib_last_error()
            lib.lbib_clear_error()
            raise LbibError(f"lbib_case_create_slab failed: {lib.lbib_error_string(rc).decode()} ({rc})")
        self.N = case.nx * case.ny * case.nz
        self.whole = x_lo == 0 and x_hi == case.nx
        self._halo = None

    @property
    def columns(self) -> slice:
        return slice(self.x_lo, self.x_hi)

    def halo(self):
        """(send_lo, send_hi, recv_lo, recv_hi) as torch CUDA tensors."""
        if self._halo is None:
            bufs = (C.c_void_p * 4)()
            n = C.c_long(0)
            _check(self.lib.lbib_slab_buffers(self.gv, bufs, C.byref(n)), "lbib_slab_buffers")
            self._halo = tuple(_tensor(bufs[i], n.value) for i in range(4))
        return self._halo

    def step_fluid(self) -> int:
        par = self.lib.lbib_slab_step_fluid(self.gv)
        _check(min(par, 0), "lbib_slab_step_fluid")
        return par

    def step_moments(self) -> None:
        _check(self.lib.lbib_slab_step_moments(self.gv), "lbib_slab_step_moments")

    def moment_tiles(self):
        """This step's moment tiles as a torch CUDA tensor (waits for the
        slab's stream); raises on a failed step (sheet out of the grid)."""
        p = C.c_void_p(0)
        n = C.c_long(0)
        _check(self.lib.lbib_slab_moments(self.gv, C.byref(p), C.byref(n)), "lbib_slab_moments")
        return _tensor(p.value, n.value) if n.value else None

    def step_move(self) -> None:
        _check(self.lib.lbib_slab_step_move(self.gv), "lbib_slab_step_move")


def _assemble(slabs, getter):
    """Whole-grid arrays from the slabs' own columns."""
    parts = [getter(s) for s in slabs]
    one = isinstance(parts[0], np.ndarray)
    outs = [np.empty_like(a) for a in ([parts[0]] if one else parts[0])]
    for s, p in zip(slabs, parts):
        for o, a in zip(outs, [p] if one else p):
            o[..., s.columns] = a[..., s.columns]
    return outs[0] if one else outs


class LocalSlabs:
    """All slabs of `case` in this process, slab k on device devices[k % len]."""

    def __init__(self, case, n: int = 2, bounds=None, devices: Sequence[int] = (0,)):
        import torch
        self.bounds = bounds or slab_bounds(case.nx, n)
        self.devices = list(devices)
        self.slabs = []
        for k, (lo, hi) in enumerate(self.bounds):
            with torch.cuda.device(self.devices[k % len(self.devices)]):
                self.slabs.append(SlabSolver(case, lo, hi))

    def close(self) -> None:
        for s in self.slabs:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def step(self) -> None:
        import torch
        S = self.slabs
        if len(S) == 1:
            S[0].run(1)
            return
        for s in S:
            s.step_fluid()
        for s in S:
            s.synchronize()
        for a, b in zip(S[:-1], S[1:]):       # a's right face meets b's left face
            ha, hb = a.halo(), b.halo()
            hb[2].copy_(ha[1].to(hb[2].device))
            ha[3].copy_(hb[0].to(ha[3].device))
        self._sync()
        for s in S:
            s.step_moments()
        U = [s.moment_tiles() for s in S]
        if U[0] is not None:
            total = U[0].clone()
            for u in U[1:]:
                total += u.to(total.device)
            for u in U:
                u.copy_(total.to(u.device))
            self._sync()
        for s in S:
            s.step_move()

    def _sync(self) -> None:
        import torch
        for d in sorted(set(self.devices)):
            torch.cuda.synchronize(d)

    def run(self, nsteps: int) -> None:
        for _ in range(nsteps):
            self.step()

    def sheet(self, k: int = 0) -> np.ndarray:
        return self.slabs[0].sheet(k)

    def df1(self) -> np.ndarray:
        return _assemble(self.slabs, lambda s: s.df1())

    def moments(self):
        return _assemble(self.slabs, lambda s: s.moments())


class DistSlabs:
    """One slab per rank of the default torch.distributed group (rank r holds
    slab r of slab_bounds(nx, world)).  `slab` may be given (any object with
    halo / step_fluid / step_moments / moment_tiles / step_move) so that the
    exchange logic can run without a GPU."""

    def __init__(self, case=None, slab=None, bounds=None):
        import torch.distributed as dist
        self.dist = dist
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.backend = dist.get_backend()
        if slab is None:
            self.bounds = bounds or slab_bounds(case.nx, self.world)
            lo, hi = self.bounds[self.rank]
            slab = SlabSolver(case, lo, hi)
        self.slab = slab

    def close(self) -> None:
        if hasattr(self.slab, "close"):
            self.slab.close()

    def _exchange(self, sends, recvs) -> None:
        """Faces: send_lo <-> rank-1, send_hi <-> rank+1 (all posted, then
        waited for, so no order of the ranks can deadlock)."""
        dist = self.dist
        pairs = []
        if self.rank > 0:
            pairs.append((sends[0], recvs[0], self.rank - 1))
        if self.rank < self.world - 1:
            pairs.append((sends[1], recvs[1], self.rank + 1))
        if not pairs:
            return
        if self.backend == "nccl":
            ops = []
            for snd, rcv, peer in pairs:
                ops += [dist.P2POp(dist.isend, snd, peer), dist.P2POp(dist.irecv, rcv, peer)]
            reqs = dist.batch_isend_irecv(ops)
        else:
            reqs = []
            for snd, rcv, peer in pairs:
                reqs += [dist.isend(snd, peer), dist.irecv(rcv, peer)]
        for r in reqs:
            r.wait()

    def step(self) -> None:
        import torch
        s, dist = self.slab, self.dist
        if getattr(s, "whole", False):         # one rank: the plain path
            s.run(1)
            return
        nccl = self.backend == "nccl"
        ctx = torch.cuda.stream(torch.cuda.ExternalStream(s.stream)) if nccl else _Null()
        with ctx:
            s.step_fluid()
            send_lo, send_hi, recv_lo, recv_hi = s.halo()
            if nccl:
                self._exchange((send_lo, send_hi), (recv_lo, recv_hi))
            else:                              # gloo: through host memory
                if hasattr(s, "synchronize"):
                    s.synchronize()
                hs = [t.cpu() for t in (send_lo, send_hi)]
                hr = [torch.empty_like(h) for h in hs]
                self._exchange(hs, hr)
                if self.rank > 0:
                    recv_lo.copy_(hr[0])
                if self.rank < self.world - 1:
                    recv_hi.copy_(hr[1])
                if recv_lo.is_cuda:
                    torch.cuda.synchronize()
            s.step_moments()
            U = s.moment_tiles()
            if U is not None:
                if nccl or not U.is_cuda:
                    dist.all_reduce(U, op=dist.ReduceOp.SUM)
                else:
                    h = U.cpu()
                    dist.all_reduce(h, op=dist.ReduceOp.SUM)
                    U.copy_(h)
                    torch.cuda.synchronize()
            s.step_move()

    def run(self, nsteps: int) -> None:
        for _ in range(nsteps):
            self.step()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def _case(a):
    from types import SimpleNamespace as NS
    w, h = 0.5 * (a.cols - 1), 0.5 * (a.rows - 1)
    sheet = NS(rows=a.rows, cols=a.cols, width=w, height=h, x0=a.x0,
               y0=(a.ny - 1) / 2.0 - h / 2.0, z0=(a.nz - 1) / 2.0 - w / 2.0)
    return NS(nx=a.nx, ny=a.ny, nz=a.nz, cube_size=4, tau=0.6, u_l=0.01, Ks_l=0.05, Kb_l=0.005,
              compat=lbib.COMPAT_ALL, sheets=[sheet])


def main(argv=None) -> int:
    """Time the slab decomposition.  Under torch.distributed.run (one rank per
    GPU, NCCL): one slab per rank, CUDA-event time on each slab's stream, max
    over ranks.  With --local N: N slabs in this process on one GPU (the
    host-synchronised transport, wall-clock per step), compared bit for bit
    with the whole grid run alongside."""
    import argparse
    import json
    import os
    import time

    import torch

    ap = argparse.ArgumentParser(description="x-slab decomposition timing")
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--nz", type=int, default=256)
    ap.add_argument("--rows", type=int, default=208)
    ap.add_argument("--cols", type=int, default=208)
    ap.add_argument("--x0", type=float, default=80.0)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--local", type=int, default=0, help="N slabs in one process on one GPU")
    a = ap.parse_args(argv)
    case = _case(a)
    cells = a.nx * a.ny * a.nz
    out = {"lattice": [a.nx, a.ny, a.nz], "sheet": [a.rows, a.cols], "steps": a.steps, "warmup": a.warmup}
    if a.local:
        L = LocalSlabs(case, n=a.local)
        L.run(a.warmup)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.run(a.steps)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3 / a.steps
        with lbib.Solver(case) as W:
            W.run(a.warmup)
            W.synchronize()
            t0 = time.perf_counter()
            W.run(a.steps)
            W.synchronize()
            wms = (time.perf_counter() - t0) * 1e3 / a.steps
            same = bool(np.array_equal(W.sheet(), L.sheet()))
        L.close()
        out.update(mode="local", slabs=a.local, bounds=L.bounds, ms_per_step=ms, mlups=cells / ms / 1e3,
                   whole_ms_per_step=wms, whole_mlups=cells / wms / 1e3, sheet_bit_identical=same)
        print(json.dumps(out))
        return 0 if same else 1
    import datetime
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local))
    D = DistSlabs(case)
    D.run(a.warmup)
    s = torch.cuda.ExternalStream(D.slab.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    e0.record(s)
    D.run(a.steps)
    e1.record(s)
    e1.synchronize()
    t = torch.tensor([e0.elapsed_time(e1) / a.steps], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    if D.rank == 0:
        out.update(mode="nccl", slabs=D.world, bounds=slab_bounds(a.nx, D.world), ms_per_step=ms,
                   mlups=cells / ms / 1e3)
        print(json.dumps(out))
    D.close()
    dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
