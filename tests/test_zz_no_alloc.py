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


def _call(fn, nodes, case, dev, stream=None):
    """One call on `stream` (a torch.cuda.Stream, or None: the legacy default
    stream); the buffers are made on that stream so the call sees them."""
    n = case.nx * case.ny * case.nz
    with torch.cuda.stream(stream if stream is not None else torch.cuda.default_stream(dev)):
        d_nodes = torch.from_numpy(np.ascontiguousarray(nodes)).to(dev)
        out = torch.full((3, n), float("nan"), dtype=torch.float64, device=dev)
        rc = fn(d_nodes.data_ptr(), nodes.shape[0], case.nx, case.ny, case.nz,
                out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(),
                None if stream is None else stream.cuda_stream)
        got = out.cpu().numpy().reshape(3, case.nz, case.ny, case.nx)
    return rc, got


def test_noalloc_spread_equals_gv_spread_twice(gpu):
    nx, ny, nz = 40, 16, 16
    case = Case(nx, ny, nz, [centred_sheet(nx, ny, nz, 6, 6, 0.5, 9.0), centred_sheet(nx, ny, nz, 8, 4, 0.5, 24.0)])
    dev = torch.device("cuda", 0)
    fn = _entry()
    s = lbib.Solver(case)
    side = torch.cuda.Stream(dev)
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
        # the same on a caller's own (non-default) stream
        rc, got = _call(fn, nodes, case, dev, stream=side)
        assert rc == 0, f"call {call} on a side stream: {rc}"
        for a, b in zip(got, ref):
            np.testing.assert_array_equal(a, b)
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
    # NaN and huge coordinates are outside the grid too (tested on the double,
    # not after an int conversion that would map NaN to 0)
    for v in (float("nan"), 1e300, -1e300, float("inf")):
        bad = nodes.copy()
        bad[5, 1] = v
        rc, got = _call(fn, bad, case, dev)
        assert rc == E_STENCIL, v
        assert not np.any(got), v
    # the regular entry point's result is back after an error
    rc, got = _call(fn, nodes, case, dev)
    assert rc == 0 and np.count_nonzero(got[0]) == 0   # zero elastic force: zero spread
