"""The x-slab decomposition's host side on the CPU: slab bounds, argument
checks before any GPU call, and the exchange protocol of DistSlabs run as
gloo ranks (2 and 3) over stand-in slabs whose buffers are CPU tensors."""
import ctypes
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

import lbib
import slabs


def test_bounds_are_whole_tiles_and_cover_the_grid():
    for nx, n in [(128, 2), (128, 3), (512, 8), (64, 16), (48, 5)]:
        b = slabs.slab_bounds(nx, n)
        assert b[0][0] == 0 and b[-1][1] == nx and len(b) == n
        assert all(lo % 4 == 0 and hi % 4 == 0 and hi - lo >= 4 for lo, hi in b)
        assert all(b[i][1] == b[i + 1][0] for i in range(n - 1))
        assert max(hi - lo for lo, hi in b) - min(hi - lo for lo, hi in b) <= 4
    for nx, n in [(128, 0), (128, 33), (130, 2)]:
        with pytest.raises(lbib.LbibError):
            slabs.slab_bounds(nx, n)


def test_slab_arguments_checked_before_any_gpu_call(lbib_built):
    lib = lbib.load()
    slabs._bind(lib)
    one_i = (ctypes.c_int * 1)(4)
    one_d = (ctypes.c_double * 1)(1.0)
    lib.lbib_clear_error()
    for lo, hi in [(2, 64), (0, 66), (0, 132), (64, 66), (64, 64), (-4, 64)]:
        gv = lib.lbib_case_create_slab(128, 16, 16, 4, 1, one_i, one_i, one_d, one_d, one_d, one_d, one_d,
                                       0.6, 0.01, 0.05, 0.005, 7, lo, hi)
        assert not gv, (lo, hi)
        assert lib.lbib_last_error() == -1
        lib.lbib_clear_error()
    bufs = (ctypes.c_void_p * 4)()
    n = ctypes.c_long(0)
    assert lib.lbib_slab_buffers(None, bufs, ctypes.byref(n)) == -1
    lib.lbib_clear_error()
    for f in ("lbib_slab_step_fluid", "lbib_slab_step_moments", "lbib_slab_step_move",
              "lbib_slab_step_fluid_direct", "lbib_slab_step_moments_direct"):
        assert getattr(lib, f)(None) == -1
        lib.lbib_clear_error()
    a = (ctypes.c_void_p * 1)(None)
    assert lib.lbib_slab_connect(None, None, 0, 0, 0, None, 0, 0, 0, 1, a, a) == -1
    assert lib.lbib_ipc_handle(None, None) == -1 and lib.lbib_ipc_open(None, None) == -1
    assert lib.lbib_ipc_close(None) == -1
    lib.lbib_clear_error()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class FakeSlab:
    """Stand-in for SlabSolver: face buffers and moment tiles as CPU
    tensors, and a record of what each phase saw."""

    def __init__(self, rank, world, n=6, tiles=5):
        import torch
        self.rank, self.world = rank, world
        self.bufs = tuple(torch.zeros(n, dtype=torch.float64) for _ in range(4))
        self.U = torch.full((tiles,), -0.0, dtype=torch.float64)
        self.log = []
        self.step = 0

    def halo(self):
        return self.bufs

    def step_fluid(self):
        self.bufs[0].fill_(100 * self.rank + 10 * self.step + 1)    # to the left neighbour
        self.bufs[1].fill_(100 * self.rank + 10 * self.step + 2)    # to the right neighbour
        self.bufs[2].fill_(float("nan"))
        self.bufs[3].fill_(float("nan"))
        return self.step & 1

    def step_moments(self):
        self.log.append(("recv", self.bufs[2][0].item(), self.bufs[3][0].item()))
        self.U.fill_(-0.0)
        self.U[self.rank] = 1000.0 * (self.rank + 1) + self.step    # owned tile
        if self.rank == 0:
            self.U[self.world] = 0.0                                # an owned +0.0
            self.U[self.world + 1] = -0.0                           # an owned -0.0

    def moment_tiles(self):
        return self.U

    def step_move(self):
        self.log.append(("U", self.U.tolist()))
        self.step += 1


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(ROOT, "distributed-lb-ib_b200"))
    import datetime
    import torch.distributed as dist
    import slabs as S
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    fake = FakeSlab(rank, world)
    d = S.DistSlabs(slab=fake)
    d.run(2)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, fake.log))


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_protocol_gloo(world):
    import math
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        log = out[r]
        for step in range(2):
            _, lo, hi = log[2 * step]
            # recv_lo holds the left neighbour's send_hi, recv_hi the right's send_lo
            if r > 0:
                assert lo == 100 * (r - 1) + 10 * step + 2
            else:
                assert math.isnan(lo)
            if r < world - 1:
                assert hi == 100 * (r + 1) + 10 * step + 1
            else:
                assert math.isnan(hi)
            _, U = log[2 * step + 1]
            want = [1000.0 * (k + 1) + step for k in range(world)]
            assert U[:world] == want
            # owned zeros keep their sign through the sum
            assert math.copysign(1.0, U[world]) == 1.0 and math.copysign(1.0, U[world + 1]) == -1.0
