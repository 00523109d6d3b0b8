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
    vp, lp, ip = C.POINTER(C.c_void_p), C.POINTER(C.c_long), C.POINTER(C.c_int)
    lib.lbib_slab_storage.argtypes = [C.c_void_p, vp, lp, ip, ip, vp, vp]
    lib.lbib_slab_connect.argtypes = [C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_int,
                                      C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_int, vp, vp]
    for n in ("lbib_slab_step_fluid_direct", "lbib_slab_step_moments_direct", "lbib_slab_check"):
        getattr(lib, n).argtypes = [C.c_void_p]
    lib.lbib_peer_access.argtypes = [C.c_int, C.c_int]
    lib.lbib_ipc_handle.argtypes = [C.c_void_p, C.c_void_p]
    lib.lbib_ipc_open.argtypes = [C.c_void_p, vp]
    lib.lbib_ipc_close.argtypes = [C.c_void_p]
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

    # ---- direct exchange (the slabs' kernels write into each other's memory)

    def storage(self) -> dict:
        """Device pointers of the populations and both moment-tile buffers,
        and the populations' geometry (after the sheet is uploaded)."""
        f, U0, U1 = C.c_void_p(0), C.c_void_p(0), C.c_void_p(0)
        Ns, sx, gx0 = C.c_long(0), C.c_int(0), C.c_int(0)
        _check(self.lib.lbib_slab_storage(self.gv, C.byref(f), C.byref(Ns), C.byref(sx), C.byref(gx0),
                                          C.byref(U0), C.byref(U1)), "lbib_slab_storage")
        return {"f": f.value, "Ns": Ns.value, "sx": sx.value, "gx0": gx0.value, "U0": U0.value, "U1": U1.value}

    def connect(self, lo, hi, U0s, U1s) -> None:
        """lo / hi: the neighbours' storage dicts (with "f" usable from this
        slab's device) or None; U0s / U1s: every slab's moment-tile buffers."""
        n = len(U0s)
        a0 = (C.c_void_p * n)(*U0s)
        a1 = (C.c_void_p * n)(*U1s)
        z = {"f": None, "Ns": 0, "sx": 0, "gx0": 0}
        lo, hi = lo or z, hi or z
        _check(self.lib.lbib_slab_connect(self.gv, lo["f"], lo["Ns"], lo["sx"], lo["gx0"], hi["f"], hi["Ns"],
                                          hi["sx"], hi["gx0"], n, a0, a1), "lbib_slab_connect")

    def step_fluid_direct(self) -> int:
        par = self.lib.lbib_slab_step_fluid_direct(self.gv)
        _check(min(par, 0), "lbib_slab_step_fluid_direct")
        return par

    def step_moments_direct(self) -> None:
        _check(self.lib.lbib_slab_step_moments_direct(self.gv), "lbib_slab_step_moments_direct")

    def check(self) -> None:
        _check(self.lib.lbib_slab_check(self.gv), "lbib_slab_check")


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

    def __init__(self, case, n: int = 2, bounds=None, devices: Sequence[int] = (0,), direct: bool = False):
        import torch
        self.bounds = bounds or slab_bounds(case.nx, n)
        self.devices = list(devices)
        self.slabs = []
        for k, (lo, hi) in enumerate(self.bounds):
            with torch.cuda.device(self.devices[k % len(self.devices)]):
                self.slabs.append(SlabSolver(case, lo, hi))
        self.direct = direct and len(self.slabs) > 1
        if self.direct:
            lib = self.slabs[0].lib
            devs = sorted(set(self.devices[:len(self.slabs)]))
            for a in devs:
                for b in devs:
                    _check(lib.lbib_peer_access(a, b), "lbib_peer_access")
            st = [s.storage() for s in self.slabs]
            U0s, U1s = [x["U0"] for x in st], [x["U1"] for x in st]
            for k, s in enumerate(self.slabs):
                s.connect(st[k - 1] if k > 0 else None, st[k + 1] if k + 1 < len(st) else None, U0s, U1s)

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
        if self.direct:
            for s in S:
                s.step_fluid_direct()
            for s in S:
                s.synchronize()
            for s in S:
                s.step_moments_direct()
            for s in S:
                s.check()                      # waits for the stream
            for s in S:
                s.step_move()
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

    def __init__(self, case=None, slab=None, bounds=None, direct: bool = False):
        import torch.distributed as dist
        self.dist = dist
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.backend = dist.get_backend()
        if slab is None:
            self.bounds = bounds or slab_bounds(case.nx, self.world)
            lo, hi = self.bounds[self.rank]
            slab = SlabSolver(case, lo, hi)
        self.slab = slab
        self.direct = direct and self.world > 1
        self._opened = []
        if self.direct:
            self._connect_ipc()

    def _connect_ipc(self) -> None:
        """Map the neighbours' populations and every slab's moment tiles into
        this process (CUDA IPC) and wire the slab to them."""
        lib = self.slab.lib
        st = self.slab.storage()
        def handle(ptr):
            h = C.create_string_buffer(64)
            _check(lib.lbib_ipc_handle(ptr, h), "lbib_ipc_handle")
            return h.raw
        mine = dict(st, hf=handle(st["f"]), hU0=handle(st["U0"]), hU1=handle(st["U1"]))
        allst = [None] * self.world
        self.dist.all_gather_object(allst, mine)
        def open_(h):
            p = C.c_void_p(0)
            _check(lib.lbib_ipc_open(h, C.byref(p)), "lbib_ipc_open")
            self._opened.append(p.value)
            return p.value
        U0s, U1s = [], []
        for r, x in enumerate(allst):
            if r == self.rank:
                U0s.append(st["U0"]); U1s.append(st["U1"])
            else:
                U0s.append(open_(x["hU0"])); U1s.append(open_(x["hU1"]))
        nb = {}
        for side, r in (("lo", self.rank - 1), ("hi", self.rank + 1)):
            if 0 <= r < self.world:
                nb[side] = dict(allst[r], f=open_(allst[r]["hf"]))
        self.slab.connect(nb.get("lo"), nb.get("hi"), U0s, U1s)

    def close(self) -> None:
        if self._opened:
            lib = self.slab.lib
            self.dist.barrier()                # no slab writes into a mapping any more
            for p in self._opened:
                lib.lbib_ipc_close(p)
            self._opened = []
            self.dist.barrier()                # every mapping closed before any slab frees its memory
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
        if self.direct:
            s.step_fluid_direct()
            s.synchronize()
            dist.barrier()
            s.step_moments_direct()
            s.check()                          # waits for the stream
            dist.barrier()
            s.step_move()
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
    ap.add_argument("--direct", action="store_true",
                    help="slabs write faces and moment tiles into each other's memory (peer / IPC pointers)")
    a = ap.parse_args(argv)
    case = _case(a)
    cells = a.nx * a.ny * a.nz
    out = {"lattice": [a.nx, a.ny, a.nz], "sheet": [a.rows, a.cols], "steps": a.steps, "warmup": a.warmup}
    if a.local:
        L = LocalSlabs(case, n=a.local, direct=a.direct)
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
        out.update(mode="local", direct=bool(a.direct), slabs=a.local, bounds=L.bounds, ms_per_step=ms, mlups=cells / ms / 1e3,
                   whole_ms_per_step=wms, whole_mlups=cells / wms / 1e3, sheet_bit_identical=same)
        print(json.dumps(out))
        return 0 if same else 1
    import datetime
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", local))
    D = DistSlabs(case, direct=a.direct)
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
        out.update(mode="nccl", direct=bool(a.direct), slabs=D.world, bounds=slab_bounds(a.nx, D.world), ms_per_step=ms,
                   mlups=cells / ms / 1e3)
        print(json.dumps(out))
    D.close()
    dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
