"""The oracle is pinned against the reference before anything is checked
against the oracle.

* bit for bit against the committed fixtures (made by running the reference,
  tests/golden/make_golden.py);
* bit for bit against the reference itself, step by step and stage by
  stage, when oracle/_ref is built (it needs the reference checkout);
* the correctly-rounded-cosine build stays within the 1e-10 relative tolerance of
  the reference.
"""
import os

import numpy as np
import pytest

import pyoracle as P
from cases import SMALL_CASES, c0_case, small_case
from pyoracle import Case, Sheet

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not P.reference_available(),
                               reason="oracle/_ref not built (needs the reference checkout)")
TOL = 1e-10


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("name", list(SMALL_CASES))
def test_oracle_matches_golden_bitwise(oracle_built, name):
    case, _ = SMALL_CASES[name]
    g = np.load(os.path.join(GOLDEN, f"small_{name}.npz"))
    o = P.Oracle(case)
    o.run(int(g["steps"]))
    for k, a in zip(["rho", "ux", "uy", "uz"], o.moments()):
        np.testing.assert_array_equal(a, g[k], err_msg=k)
    np.testing.assert_array_equal(o.sheet(), g["sheet"])


@pytest.mark.parametrize("name", list(SMALL_CASES))
def test_oracle_cr_cosine_within_tolerance(oracle_built, name):
    case, _ = SMALL_CASES[name]
    g = np.load(os.path.join(GOLDEN, f"small_{name}.npz"))
    o = P.Oracle(case, cr_cos=True)
    o.run(int(g["steps"]))
    rho, ux, uy, uz = o.moments()
    assert rel_l2(rho, g["rho"]) <= TOL
    assert rel_l2(np.stack([ux, uy, uz]), np.stack([g["ux"], g["uy"], g["uz"]])) <= TOL
    assert rel_l2(o.sheet()[..., :3], g["sheet"][..., :3]) <= TOL


@needs_ref
@pytest.mark.parametrize("name", list(SMALL_CASES))
def test_oracle_matches_reference_every_step(oracle_built, name):
    case, steps = SMALL_CASES[name]
    o, r = P.Oracle(case), P.Reference(case)
    for _ in range(min(steps, 12)):
        o.run(1); r.run(1)
        for a, b in zip(o.moments(), r.moments()):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(o.df(0), r.df(0))
        np.testing.assert_array_equal(o.df(1), r.df(1))
        np.testing.assert_array_equal(o.sheet(), r.sheet())


@needs_ref
def test_oracle_stages_match_reference(oracle_built):
    """Every stage alone, on a deformed sheet and a developed flow."""
    case, _ = SMALL_CASES["wall"]
    o, r = P.Oracle(case), P.Reference(case)
    o.run(6); r.run(6)
    rng = np.random.default_rng(3)
    sh = r.sheet().copy()
    sh[..., :3] += rng.uniform(-0.3, 0.3, size=sh[..., :3].shape)
    o.set_sheet(0, sh); r.set_sheet(0, sh)
    for st in ["bending", "stretching", "elastic", "spread", "collide", "stream", "bounceback",
               "moments", "move", "copy_inout", "replace"]:
        assert o.stage(st) == 0 and r.stage(st) == 0
        np.testing.assert_array_equal(o.sheet(), r.sheet(), err_msg=st)
        for a, b in zip(o.force(), r.force()):
            np.testing.assert_array_equal(a, b, err_msg=st)
        for a, b in zip(o.moments(), r.moments()):
            np.testing.assert_array_equal(a, b, err_msg=st)
        np.testing.assert_array_equal(o.df(0), r.df(0), err_msg=st)
        np.testing.assert_array_equal(o.df(1), r.df(1), err_msg=st)


@needs_ref
def test_oracle_matches_reference_random_sheet(oracle_built):
    """Bending/stretching ends, odd sizes and a crumpled sheet."""
    case = Case(32, 24, 16, [Sheet(9, 7, 3.0, 4.0, 10.5, 9.3, 5.2)], Ks_l=0.2, Kb_l=0.02)
    o, r = P.Oracle(case), P.Reference(case)
    rng = np.random.default_rng(11)
    sh = r.sheet().copy()
    sh[..., :3] += rng.normal(0, 0.4, size=sh[..., :3].shape)
    o.set_sheet(0, sh); r.set_sheet(0, sh)
    o.run(8); r.run(8)
    for a, b in zip(o.moments(), r.moments()):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(o.sheet(), r.sheet())


def test_compat_bits(oracle_built):
    """The reference's loop-bound slips only act when num_cubes_x <
    num_cubes_z; the bending slip acts always."""
    base, steps = SMALL_CASES["base"]
    xltz, steps2 = SMALL_CASES["xltz"]

    def run(case, compat, n):
        c = Case(case.nx, case.ny, case.nz, case.sheets, case.tau, case.u_l, case.Ks_l, case.Kb_l,
                 case.cube_size, compat)
        o = P.Oracle(c)
        o.run(n)
        return o.moments()[1]
    ref = run(base, P.COMPAT_ALL, 10)
    np.testing.assert_array_equal(ref, run(base, P.COMPAT_BEND_X_BUG, 10))
    assert not np.array_equal(ref, run(base, P.COMPAT_ALL & ~P.COMPAT_BEND_X_BUG, 10))
    ref2 = run(xltz, P.COMPAT_ALL, 10)
    assert not np.array_equal(ref2, run(xltz, P.COMPAT_ALL & ~P.COMPAT_YWALL_CUBES_X, 10))
    assert not np.array_equal(ref2, run(xltz, P.COMPAT_ALL & ~P.COMPAT_INOUT_PTHREAD, 10))


def test_oracle_stencil_error(oracle_built):
    case = small_case(24, 12, 12, 6, 6, 8.0)
    o = P.Oracle(case)
    sh = o.sheet().copy()
    sh[..., 0] = 0.5
    o.set_sheet(0, sh)
    with pytest.raises(RuntimeError):
        o.run(1)


@pytest.mark.slow
def test_oracle_c0_1000_matches_golden(oracle_built):
    """The reference's workload for 1000 steps, bit for bit (OpenMP oracle)."""
    path = os.path.join(GOLDEN, "c0_1000.npz")
    g = np.load(path)
    case = c0_case()
    P.Oracle.set_threads(os.cpu_count() or 1)
    o = P.Oracle(case)
    o.run(int(g["steps"]))
    rho, ux, uy, uz = o.moments()
    idx = g["sample_idx"]
    np.testing.assert_array_equal(o.sheet(), g["sheet"])
    for a, k in zip([rho, ux, uy, uz], ["rho", "ux", "uy", "uz"]):
        np.testing.assert_array_equal(a.ravel()[idx], g[k])
    norms = np.array([np.linalg.norm(rho), np.linalg.norm(ux), np.linalg.norm(uy), np.linalg.norm(uz)])
    np.testing.assert_array_equal(norms, g["norms"])
