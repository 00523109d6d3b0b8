"""The physics options on the GPU (LBIB_OPT_*; no reference counterpart --
the benchmark workloads ask for them and the reference has none of them):
bit for bit against the oracle built with the same options and cosine
(liboracle_cr.so), through both fluid paths (two-cell rows and the generic
kernel), over both AA parities.  The oracle's option code is pinned by its
own property tests (tests/test_oracle_options.py); the parity of these
options against the reference itself is unpinned -- the reference has no
such physics.  The low-precision forms run the options too and stay within
their usual distance of the FP64 solution."""
import numpy as np
import pytest

import lbib
import pyoracle as P
from pyoracle import Case, Sheet
from test_gpu_parity import assert_same_state

pytestmark = pytest.mark.gpu
PER, REST, PIN = 0x100, 0x200, 0x400

OPT_CASES = {
    "periodic_z": (Case(24, 12, 20, [Sheet(6, 6, 2.5, 2.5, 8.0, 3.5, 8.25)], compat=P.COMPAT_ALL | PER), 14),
    # a sheet whose stencil reaches the cells next to z = 2: the wrapped links act on it
    "periodic_z_low": (Case(24, 12, 16, [Sheet(6, 6, 2.5, 2.5, 8.0, 4.0, 3.25)], compat=PER), 12),
    "rest_start": (Case(24, 12, 12, [Sheet(6, 6, 2.5, 2.5, 8.0, 3.5, 3.5)], compat=P.COMPAT_ALL | REST), 14),
    "pinned_row": (Case(24, 12, 12, [Sheet(6, 6, 2.5, 2.5, 8.0, 3.5, 3.5)], compat=P.COMPAT_ALL | PIN), 14),
    "all_three": (Case(32, 16, 20, [Sheet(8, 8, 3.5, 3.5, 10.0, 5.5, 8.25)],
                       compat=P.COMPAT_ALL | PER | REST | PIN), 12),
    "two_sheets_pinned": (Case(40, 16, 16, [Sheet(6, 6, 2.5, 2.5, 9.0, 5.0, 5.0), Sheet(8, 4, 1.5, 3.5, 24.0, 4.0, 6.0)],
                               compat=P.COMPAT_ALL | PIN | PER), 10),
}


@pytest.fixture(params=["two_cell", "generic"])
def fluid_path(request, monkeypatch):
    if request.param == "generic":
        monkeypatch.setenv("LBIB_FLUID_BULK", "0")
    else:
        monkeypatch.delenv("LBIB_FLUID_BULK", raising=False)
    return request.param


@pytest.mark.parametrize("name", sorted(OPT_CASES))
def test_options_bitexact_vs_oracle_cr(gpu, oracle_built, fluid_path, name):
    case, steps = OPT_CASES[name]
    s = lbib.Solver(case)
    o = P.Oracle(case, cr_cos=True)
    assert_same_state(s, o, case)
    s.run(1); o.run(1)
    assert_same_state(s, o, case)
    s.run(steps - 1); o.run(steps - 1)
    assert_same_state(s, o, case)
    s.close()


def test_pinned_row_stays_and_rest_start_fills_the_channel(gpu):
    case, steps = OPT_CASES["all_three"]
    with lbib.Solver(case) as s:
        s0 = s.sheet().copy()
        ux0 = s.moments()[1]
        assert np.all(ux0[:, :, 3:-3] == 0.0)
        s.run(steps)
        s1 = s.sheet()
        np.testing.assert_array_equal(s1[0, :, :3], s0[0, :, :3])
        assert np.abs(s1[1:, :, :3] - s0[1:, :, :3]).max() > 0
        assert s.moments()[1][10, 8, 3] > 0            # the inflow has entered


@pytest.mark.parametrize("prec,tol", [("f32", 1e-4), ("f16-flow", 2e-2)])
def test_options_in_low_precision(gpu, prec, tol):
    case, steps = OPT_CASES["all_three"]
    with lbib.Solver(case) as a, lbib.Solver(case, prec) as b:
        a.run(steps); b.run(steps)
        ua, ub = np.stack(a.moments()[1:]), np.stack(b.moments()[1:])
        sl = (slice(None), slice(2, -2), slice(2, -2), slice(2, -2))
        assert np.linalg.norm(ub[sl] - ua[sl]) <= tol * np.linalg.norm(ua[sl])
        np.testing.assert_array_equal(b.sheet()[0, :, :3], a.sheet()[0, :, :3])   # pinned in both
