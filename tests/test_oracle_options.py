"""The oracle's physics options (no reference counterpart: the benchmark
workloads ask for them, the reference has none of them): properties that
pin the restatement's option code without the reference.

* LBIB_OPT_PERIODIC_Z: the problem is invariant under a shift by 4 cells
  in z on the z-torus, so shifting the sheet shifts the whole solution by
  4 cells -- to rounding: the bending force combines absolute positions
  (-X[j+2] + 4 X[j+1] - 6 X[j] ...), whose partial sums round differently
  4 cells apart, so the bar is 1e-12 relative, far below what a wrong wrap
  would give -- and the cells next to z = 2, nz-3 see the other side
  instead of a wall.
* LBIB_OPT_REST_START: the interior starts at u = 0, the planes at u_l.
* LBIB_OPT_PIN_ROW0: row 0 does not move, the others do.
"""
import numpy as np

import pyoracle as P
from pyoracle import Case, Sheet

PER, REST, PIN = 0x100, 0x200, 0x400


def _case(opts, z0=8.25, nz=20):
    return Case(24, 12, nz, [Sheet(6, 6, 2.5, 2.5, 8.0, 3.5, z0)], compat=P.COMPAT_ALL | opts)


def test_periodic_z_is_translation_invariant():
    a = P.Oracle(_case(PER))
    b = P.Oracle(_case(PER, z0=12.25))       # the same sheet, 4 cells further in z
    a.run(12)
    b.run(12)
    ra, ua = a.moments()[0], a.moments()[1]
    rb, ub = b.moments()[0], b.moments()[1]
    nz = 20
    I = np.arange(2, nz - 2)                  # z of the interior, period nz - 4
    shifted = 2 + (I - 2 + 4) % (nz - 4)
    for fa, fb in [(ra, rb), (ua, ub)]:
        x, y = fa[I, 2:-2, 2:-2], fb[shifted, 2:-2, 2:-2]
        assert np.linalg.norm(y - x) <= 1e-12 * np.linalg.norm(x)
    np.testing.assert_allclose(b.sheet()[..., 2], a.sheet()[..., 2] + 4.0, rtol=0, atol=1e-12)
    np.testing.assert_allclose(b.sheet()[..., :2], a.sheet()[..., :2], rtol=0, atol=1e-12)
    # the flow past the sheet is not uniform in z: the test is not trivial
    assert np.ptp(ua[I, 6, 10]) > 1e-6


def test_periodic_z_differs_from_walls():
    a = P.Oracle(_case(0))
    b = P.Oracle(_case(PER))
    a.run(6)
    b.run(6)
    # the cells next to the z walls see the other side instead of a wall
    assert not np.array_equal(a.moments()[1][2], b.moments()[1][2])


def test_rest_start_and_pinned_row():
    o = P.Oracle(_case(REST | PIN))
    ux = o.moments()[1]
    assert np.all(ux[:, :, 3:-3] == 0.0) and np.all(ux[:, :, 2] == 0.01) and np.all(ux[:, :, -3] == 0.01)
    s0 = o.sheet().copy()
    o.run(15)
    s1 = o.sheet()
    np.testing.assert_array_equal(s1[0, :, :3], s0[0, :, :3])
    assert np.abs(s1[1:, :, :3] - s0[1:, :, :3]).max() > 0
    # the inflow enters the channel from the inlet plane
    assert o.moments()[1][6, 6, 3] > 0
