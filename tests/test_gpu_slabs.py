"""The x-slab decomposition on the GPU: slabs advanced together (in one
process, and as two gloo ranks exchanging through host memory) give the
whole grid's run bit for bit -- sheet, populations and moments -- with the
sheet's stencil crossing a slab face."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

import lbib
import slabs
from cases import c0_case, small_case
from pyoracle import Case, Sheet

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("direct", [False, True])
@pytest.mark.parametrize("bounds", [[(0, 20), (20, 68), (68, 128)], [(0, 64), (64, 128)]])
def test_local_slabs_equal_whole_grid(gpu, bounds, direct):
    """direct: the slabs' kernels write faces and moment tiles straight into
    each other's memory; otherwise through the face buffers and a sum."""
    case, steps = c0_case(), 25
    with lbib.Solver(case) as whole:
        whole.run(steps)
        sheet, df1, mom = whole.sheet(), whole.df1(), whole.moments()
    with slabs.LocalSlabs(case, bounds=bounds, direct=direct) as L:
        L.run(steps)
        assert np.array_equal(L.sheet(), sheet)
        assert np.array_equal(L.df1()[:, 2:-2, 2:-2, 2:-2], df1[:, 2:-2, 2:-2, 2:-2])
        for a, b in zip(L.moments(), mom):
            assert np.array_equal(a, b)
        # the sheet moved, and the run reached odd and even parities
        assert np.abs(sheet[..., 0] - L.slabs[0].case.sheets[0].x0).max() > 0


def test_slab_refuses_the_whole_grid_calls(gpu, tmp_path):
    """A slab GV cannot run whole-grid steps or write restart files; a whole
    grid cannot take slab steps."""
    case = small_case(64, 16, 16, 8, 8, x0=30.0)
    s = slabs.SlabSolver(case, 0, 32)
    try:
        with pytest.raises(lbib.LbibError, match="out of order"):
            s.run(1)
        with pytest.raises(lbib.LbibError, match="out of order"):
            s.save(str(tmp_path / "r.bin"))
        with pytest.raises(lbib.LbibError, match="out of order"):
            s.step_fluid_direct()                      # not connected
    finally:
        s.close()
    w = slabs.SlabSolver(case, 0, 64)                  # the whole grid
    try:
        assert w.whole
        with pytest.raises(lbib.LbibError, match="out of order"):
            w.step_fluid()
        w.run(2)
    finally:
        w.close()


def test_a_stencil_leaving_the_grid_stops_the_slabs(gpu):
    # a sheet one cell from the outlet: its stencil leaves the grid within a few steps
    bad = Case(32, 16, 16, [Sheet(4, 4, 1.5, 1.5, 29.3, 7.0, 7.0)], u_l=0.1)
    with lbib.Solver(bad) as whole:
        with pytest.raises(lbib.LbibError, match="stencil"):
            whole.run(20)
    with slabs.LocalSlabs(bad, bounds=[(0, 16), (16, 32)]) as L:
        with pytest.raises(lbib.LbibError, match="stencil"):
            L.run(20)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _slab_case():
    return small_case(64, 16, 16, 8, 8, x0=30.0)


def _rank_main(rank, world, port, steps, q, direct=False):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    for p in (os.path.join(ROOT, "distributed-lb-ib_b200"), os.path.join(ROOT, "tests"),
              os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import datetime
    import torch.distributed as dist
    import slabs as S
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    d = S.DistSlabs(case=_slab_case(), direct=direct)
    d.run(steps)
    s = d.slab
    q.put((rank, s.x_lo, s.x_hi, s.sheet(), s.df1()[:, :, :, s.columns]))
    dist.barrier()
    d.close()
    dist.destroy_process_group()


@pytest.mark.parametrize("direct", [False, True])
def test_two_ranks_gloo_equal_whole_grid(gpu, direct):
    """Two processes on one GPU: face buffers through gloo, or (direct) each
    rank's kernels writing into the other's memory through CUDA IPC, with a
    host barrier between the phases (no kernel waits on the other rank)."""
    steps, world = 31, 2
    case = _slab_case()
    with lbib.Solver(case) as whole:
        whole.run(steps)
        sheet, df1 = whole.sheet(), whole.df1()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, steps, q, direct)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = np.zeros_like(df1)
    for rank, lo, hi, sh, part in out:
        assert np.array_equal(sh, sheet), rank
        got[:, :, :, lo:hi] = part
    assert np.array_equal(got[:, 2:-2, 2:-2, 2:-2], df1[:, 2:-2, 2:-2, 2:-2])
