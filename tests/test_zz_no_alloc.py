"""lbib_spread_force_noalloc: the force spread for hosts that cannot allocate
GPU memory while they run, checked through the C ABI against the spread of
the regular GV path (fiber_SpreadForce), on two calls in a row.

The tolerance is the one the parity tests use against the oracle: exact
equality, because both paths evaluate the same operations in the same order.
This file is collected last (test_zz_*); it needs nothing from the other
tests and passes alone in a fresh process as well as after them.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import lbib
from pyoracle import Case, Sheet, centred_sheet

pytestmark = pytest.mark.gpu

E_STENCIL = -3
E_LIMIT = -8
MAX_NODES = 1 << 18


def _entry():
    f = lbib.load().lbib_spread_force_noalloc
    f.argtypes = [C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p]
    f.restype = C.c_int
    return f


def _call(fn, nodes, case, dev):
    n = case.nx * case.ny * case.nz
    d_nodes = torch.from_numpy(np.ascontiguousarray(nodes)).to(dev)
    out = torch.full((3, n), float("nan"), dtype=torch.float64, device=dev)
    rc = fn(d_nodes.data_ptr(), nodes.shape[0], case.nx, case.ny, case.nz,
            out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), None)
    return rc, out.cpu().numpy().reshape(3, case.nz, case.ny, case.nx)


def test_noalloc_spread_equals_gv_spread_twice(gpu):
    nx, ny, nz = 40, 16, 16
    case = Case(nx, ny, nz, [centred_sheet(nx, ny, nz, 6, 6, 0.5, 9.0), centred_sheet(nx, ny, nz, 8, 4, 0.5, 24.0)])
    dev = torch.device("cuda", 0)
    fn = _entry()
    s = lbib.Solver(case)
    for call, steps in enumerate([3, 4]):
        s.run(steps)
        # the GV path's spread of the current sheet (start of the next step)
        s.stage("bending")
        s.stage("spread")
        ref = s.force()
        nodes = np.concatenate([s.sheet(k).reshape(-1, 12) for k in range(len(case.sheets))])
        rc, got = _call(fn, nodes, case, dev)
        assert rc == 0, f"call {call}: {rc}"
        for a, b in zip(got, ref):
            np.testing.assert_array_equal(a, b)
        assert np.count_nonzero(got[0]) > 0
        # finish the step the stages began
        for st in ["collide", "moments", "move"]:
            s.stage(st)
    s.close()


def test_noalloc_limits_and_errors(gpu):
    nx, ny, nz = 24, 12, 12
    case = Case(nx, ny, nz, [Sheet(6, 6, 2.5, 2.5, 8.0, 4.0, 4.0)])
    dev = torch.device("cuda", 0)
    fn = _entry()
    nodes = np.zeros((36, 12))
    nodes[:, 0], nodes[:, 1], nodes[:, 2] = 8.0, 5.0, 5.0
    # above the fixed maximum: rejected before any work
    n = nx * ny * nz
    out = torch.zeros((3, n), dtype=torch.float64, device=dev)
    d = torch.from_numpy(nodes).to(dev)
    assert fn(d.data_ptr(), MAX_NODES + 1, nx, ny, nz, out[0].data_ptr(), out[1].data_ptr(),
              out[2].data_ptr(), None) == E_LIMIT
    # a stencil outside the grid: the reference exits; here an error and zero force
    bad = nodes.copy()
    bad[3, 0] = 0.5
    rc, got = _call(fn, bad, case, dev)
    assert rc == E_STENCIL
    assert not np.any(got)
