"""Batched independent problems (lbib_batch_*) against the same problems
run one at a time through the GV path.

An FP64 batch must give every problem the bits it gets on its own (same
kernels' arithmetic, -fmad=false); the low-precision batch runs the same
word kernels and must match its one-grid runs to rounding.  A problem whose
sheet leaves its grid stops without disturbing the others.
"""
import numpy as np
import pytest

import lbib
from pyoracle import Case, Sheet, centred_sheet

pytestmark = pytest.mark.gpu


def problems():
    """Uneven sizes and physics, one sheet each."""
    return [
        Case(32, 16, 16, [centred_sheet(32, 16, 16, 8, 8, 0.5, 10.0)]),
        Case(48, 20, 24, [centred_sheet(48, 20, 24, 6, 10, 0.5, 12.0)], tau=0.7, u_l=0.02, Ks_l=0.1, Kb_l=0.001),
        Case(24, 12, 12, [centred_sheet(24, 12, 12, 6, 6, 0.5, 8.0)], tau=0.55, u_l=0.005, Ks_l=0.01, Kb_l=0.01),
        Case(160, 12, 16, [centred_sheet(160, 12, 16, 5, 7, 0.5, 30.0)], tau=0.8, u_l=0.015),
    ]


def alone(case, precision, steps):
    with lbib.Solver(case, precision) as s:
        for n in steps:
            s.run(n)
        return s.sheet(0), s.moments(), s.df1()


def interior(case):
    return (slice(None), slice(2, case.nz - 2), slice(2, case.ny - 2), slice(2, case.nx - 2))


SPLITS = [1, 4, 3, 2]   # eager first step, graph pairs, an eager tail, more pairs


def test_f64_batch_equals_problems_alone(gpu):
    cases = problems()
    with lbib.Batch(cases, "f64") as b:
        for n in SPLITS:
            b.run(n)
        got = [(b.sheet(k), b.moments(k), b.df1(k)) for k in range(len(cases))]
        codes, _ = b.status()
        assert not codes.any()
        assert b.steps == sum(SPLITS)
    for k, case in enumerate(cases):
        sh, mom, df = alone(case, "f64", SPLITS)
        np.testing.assert_array_equal(got[k][0], sh, err_msg=f"sheet {k}")
        for name, a, c in zip(["rho", "ux", "uy", "uz"], got[k][1], mom):
            np.testing.assert_array_equal(a, c, err_msg=f"{name} {k}")
        np.testing.assert_array_equal(got[k][2][interior(case)], df[interior(case)], err_msg=f"df1 {k}")


@pytest.mark.parametrize("prec", ["f16-flow", "bf16", "f32"])
def test_low_precision_batch_matches_problems_alone(gpu, prec):
    cases = problems()
    with lbib.Batch(cases, prec) as b:
        nv = b.variants()
    for v in range(nv):
        with lbib.Batch(cases, prec) as b:
            b.set_variant(v)
            for n in SPLITS:
                b.run(n)
            got = [(b.sheet(k), b.df1(k)) for k in range(len(cases))]
        for k, case in enumerate(cases):
            with lbib.Solver(case, prec) as s:
                s.set_variant(v)
                for n in SPLITS:
                    s.run(n)
                sh, df = s.sheet(0), s.df1()
            tol = {"f32": 1e-9}.get(prec, 2e-5)
            assert np.max(np.abs(got[k][1][interior(case)] - df[interior(case)])) <= tol, (v, k)
            assert np.max(np.abs(got[k][0] - sh)) <= 1e-6, (v, k)


def test_a_failing_problem_stops_alone(gpu):
    cases = problems()
    # a sheet one cell from the outlet: its stencil leaves the grid within a few steps
    bad = Case(32, 16, 16, [Sheet(4, 4, 1.5, 1.5, 29.3, 7.0, 7.0)], u_l=0.1)
    mixed = cases[:2] + [bad] + cases[2:]
    with lbib.Batch(mixed, "f64") as b:
        for n in SPLITS:
            b.run(n)
        codes, step = b.status()
        got = [b.sheet(k) for k in range(len(mixed))]
    assert codes[2] == -3 and step[2] >= 1
    assert not np.delete(codes, 2).any()
    for k, case in enumerate(cases):
        kk = k if k < 2 else k + 1
        np.testing.assert_array_equal(got[kk], alone(case, "f64", SPLITS)[0])


def test_autotune_per_size_class(gpu):
    cases = problems() + problems()[:2]
    with lbib.Batch(cases, "f16-flow") as b:
        cls, ms = b.autotune(4)
        assert ms.shape == (4, b.variants()) and (ms > 0).all()
        assert list(cls) == [0, 1, 2, 3, 0, 1]
        assert b.steps == 0
        b.run(5)
        a = b.df1(3)
    # the chosen variants, set by hand, give the same run
    with lbib.Batch(cases, "f16-flow") as b:
        for k in range(len(cases)):
            b.set_variant(int(np.argmin(ms[cls[k]])), k)
        b.run(5)
        np.testing.assert_array_equal(b.df1(3), a)


def test_pinned_leading_row_stays(gpu):
    case = problems()[0]
    p = lbib.Problem.from_case(case)
    p.pinned = 1
    with lbib.Batch([p, lbib.Problem.from_case(case)], "f64") as b:
        s0 = b.sheet(0)
        b.run(6)
        s1, free = b.sheet(0), b.sheet(1)
    np.testing.assert_array_equal(s1[0, :, :3], s0[0, :, :3])
    assert np.abs(s1[1:, :, :3] - s0[1:, :, :3]).max() > 0
    assert np.abs(free[0, :, :3] - s0[0, :, :3]).max() > 0


def test_failure_step_counts_through_graph_replays(gpu):
    """The step a problem stops at is the live step, also inside replayed graphs."""
    bad = Case(32, 16, 16, [Sheet(4, 4, 1.5, 1.5, 26.0, 7.0, 7.0)], u_l=0.1)
    with lbib.Batch([bad, problems()[0]], "f64") as b:
        b.run(80)
        codes, step = b.status()
    assert codes[0] == -3 and step[0] > 6 and codes[1] == 0
