"""Low-precision population storage against the FP64 drop-in.

The FP64 path is pinned to the oracle bit for bit (test_gpu_parity.py); the
FP32 / FP16 / BF16 forms store deviations from a shift and do FP32
arithmetic, so they are judged by their error against the FP64 solution of
the same case.  Bars (relative L2 of u over the fluid interior, tip =
mean x-displacement of the last fiber row, mass = FP64 population sum):

  form        velocity   tip      |mass - mass64| / mass64
  f32         1e-4       1e-4     1e-7
  f16-flow    1e-3       2e-3     1e-5
  f16         1e-2       5e-3     1e-5
  bf16-flow   2e-2       2e-2     1e-4
  bf16        5e-2       2e-2     2e-4

on the 128x64x64 lattice with one 52x52 sheet after 1000 steps, and the
starting state to the storage rounding.  The FP64 sums are also checked
against the oracle's populations.
"""
import numpy as np
import pytest

import lbib
import precision
import pyoracle as P
from cases import c0_case, small_case

pytestmark = pytest.mark.gpu

LP = ["f32", "f16", "bf16", "f32-flow", "f16-flow", "bf16-flow"]
# lattice velocities in the library's q order (the reference's c table,
# cube_pthread/lbm_ib.c:777-833, in internal axes)
C = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 0, 1], [0, 0, -1], [0, -1, 0], [0, 1, 0],
              [1, 0, 1], [-1, 0, -1], [1, 0, -1], [-1, 0, 1], [0, -1, 1], [0, 1, -1],
              [0, 1, 1], [0, -1, -1], [1, -1, 0], [-1, 1, 0], [1, 1, 0], [-1, -1, 0]], dtype=np.float64)
BARS = {
    "f32": (1e-4, 1e-4, 1e-7),
    "f16-flow": (1e-3, 2e-3, 1e-5),
    "f16": (1e-2, 5e-3, 1e-5),
    "bf16-flow": (2e-2, 2e-2, 1e-4),
    "bf16": (5e-2, 2e-2, 2e-4),
}
# largest |f - f64| of the initial populations: half an ulp of the stored deviation
INIT_TOL = {"f32": 1e-9, "f32-flow": 1e-9, "f16": 2e-6, "f16-flow": 1e-8, "bf16": 2e-5, "bf16-flow": 1e-7}


def interior(case):
    return (slice(None), slice(2, case.nz - 2), slice(2, case.ny - 2), slice(2, case.nx - 2))


@pytest.mark.parametrize("prec", LP)
def test_initial_populations_match_f64(gpu, prec):
    case = small_case(32, 16, 16, 8, 8, 10.0)
    with lbib.Solver(case, "f64") as s:
        ref = s.df1()[interior(case)]
    with lbib.Solver(case, prec) as s:
        got = s.df1()[interior(case)]
    assert np.max(np.abs(got - ref)) <= INIT_TOL[prec]


def test_f64_conservation_sums_match_oracle(gpu, oracle_built):
    case = small_case(24, 12, 12, 6, 6, 8.0)
    o = P.Oracle(case, cr_cos=True)
    o.run(12)
    with lbib.Solver(case) as s:
        s.run(12)
        got = s.conservation()
        again = s.conservation()
    df = o.df(0)[interior(case)]
    want = [df.sum()] + [np.tensordot(C[:, k], df, 1).sum() for k in range(3)]
    np.testing.assert_array_equal(got, again)  # fixed summation order
    assert abs(got[0] - want[0]) <= 1e-13 * abs(want[0])
    np.testing.assert_allclose(got[1:], want[1:], rtol=0, atol=1e-12 * abs(want[0]))


@pytest.mark.parametrize("prec", LP)
def test_low_precision_sums_match_populations(gpu, prec):
    case = small_case(32, 16, 16, 8, 8, 10.0)
    with lbib.Solver(case, prec) as s:
        s.run(7)
        got = s.conservation()
        df = s.df1()[interior(case)]
    assert abs(got[0] - df.sum()) <= 1e-12 * df.sum()


@pytest.fixture(scope="module")
def c0_reference(gpu):
    return precision.run_case(c0_case(), 1000, "f64")


@pytest.mark.parametrize("prec", sorted(BARS))
def test_error_against_f64_after_1000_steps(c0_reference, prec):
    case = c0_case()
    r = precision.compare(c0_reference, precision.run_case(case, 1000, prec), case)
    v, tip, mass = BARS[prec]
    assert r["velocity_rel_l2"] <= v, r
    assert r["tip_displacement_rel"] <= tip, r
    assert abs(r["mass_vs_f64"]) <= mass, r


def test_precision_switch_rebuilds_state(gpu):
    """lbib_set_precision before init_gv rebuilds the GPU state; after it, refused."""
    lib = lbib.load()
    case = small_case(32, 16, 16, 8, 8, 10.0)
    with lbib.Solver(case, "f16-flow") as s:
        lib.lbib_clear_error()
        assert lib.lbib_set_precision(s.gv, lbib.PREC_F32) == -4  # sheets already uploaded
        lib.lbib_clear_error()


# cases for the word kernel: rows of 3+ warps (lane 0 / 31 crossings), a row
# of one active word (nx = 12), forcing tiles at the row ends; for the
# TMA-staged variants, items of 16 rows (nx = 32), of 8 rows (nx = 64), of
# exactly one row (nx = 512) and rows of two segments, the second partial
# (nx = 640); rows whose word count does not divide 128 (nx = 160, 12) fall
# back to the plain word kernel
WORD_CASES = {
    "long_rows": (small_case(160, 12, 12, 6, 6, 20.0), 9),
    "short_rows": (small_case(12, 12, 24, 6, 6, 5.0), 7),
    "sheet_at_inlet": (small_case(32, 16, 16, 8, 8, 4.5), 9),
    "eight_row_items": (small_case(64, 16, 20, 8, 8, 10.0), 8),
    "one_row_items": (small_case(512, 12, 16, 6, 6, 40.0), 7),
    "two_segment_rows": (small_case(640, 12, 12, 6, 6, 20.0), 7),
}
# rounding-level differences only: FMA contraction may differ between the
# two kernels, which moves a 16-bit value by at most an ulp now and then
WORD_TOL = {"f32": 1e-9, "f32-flow": 1e-9, "f16": 2e-6, "f16-flow": 2e-6, "bf16": 2e-5, "bf16-flow": 2e-5}


def _run(case, prec, steps, monkeypatch, bulk, variant=-1):
    if bulk:
        monkeypatch.delenv("LBIB_FLUID_BULK", raising=False)
    else:
        monkeypatch.setenv("LBIB_FLUID_BULK", "0")
    with lbib.Solver(case, prec) as s:
        s.set_variant(variant)
        s.run(steps)
        return s.df1()[interior(case)], s.moments(), s.sheet(0)


@pytest.mark.parametrize("prec", LP)
@pytest.mark.parametrize("name", sorted(WORD_CASES))
def test_word_kernel_matches_cell_kernel(gpu, monkeypatch, prec, name):
    """Every variant of the multi-cell word kernel against the one-cell
    generic kernel, over both AA parities."""
    case, steps = WORD_CASES[name]
    b = _run(case, prec, steps, monkeypatch, False)
    with lbib.Solver(case, prec) as s:
        nv = s.variants()
    assert nv >= 3
    for v in range(nv):
        a = _run(case, prec, steps, monkeypatch, True, v)
        assert np.max(np.abs(a[0] - b[0])) <= WORD_TOL[prec], v
        for x, y in zip(a[1], b[1]):
            assert np.max(np.abs(x - y)) <= 50 * WORD_TOL[prec], v
        assert np.max(np.abs(a[2] - b[2])) <= 1e-6, v


def test_autotune_leaves_the_run_unchanged(gpu):
    case = small_case(64, 16, 16, 8, 8, 10.0)
    with lbib.Solver(case, "f16-flow") as s:
        best, ms = s.autotune(4)
        assert 0 <= best < s.variants() and len(ms) == s.variants() and min(ms) > 0
        s.run(6)
        a = s.df1()
    with lbib.Solver(case, "f16-flow") as s:
        s.set_variant(best)
        s.run(6)
        b = s.df1()
    np.testing.assert_array_equal(a, b)
    with lbib.Solver(case, "f16-flow") as s:
        s.run(1)
        lib = lbib.load()
        assert lib.lbib_autotune(s.gv, 4, None, 0) == -4   # only before the first step
        lib.lbib_clear_error()
