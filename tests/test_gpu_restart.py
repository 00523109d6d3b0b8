"""Restart files: save after some steps, load into a freshly set-up problem,
and the continued run equals the uninterrupted one bit for bit."""
import numpy as np
import pytest

import lbib
from cases import small_case
from pyoracle import Case, centred_sheet

pytestmark = pytest.mark.gpu


def state(s):
    return s.moments(), s.sheet(0), s.df1(), s.force()


@pytest.mark.parametrize("prec", ["f64", "f16-flow"])
@pytest.mark.parametrize("first", [7, 8])       # both AA parities at the save
def test_restart_continues_bit_for_bit(gpu, tmp_path, prec, first):
    case = small_case(32, 16, 16, 8, 8, 10.0)
    path = str(tmp_path / "run.rst")
    with lbib.Solver(case, prec) as s:
        s.run(first)
        s.save(path)
        s.run(5)
        want = state(s)
    with lbib.Solver(case, prec) as s:
        s.load(path)
        s.run(5)
        got = state(s)
    for a, b in zip(got[0], want[0]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(got[1], want[1])
    np.testing.assert_array_equal(got[2], want[2])
    for a, b in zip(got[3], want[3]):
        np.testing.assert_array_equal(a, b)


def test_restart_refuses_another_grid(gpu, tmp_path):
    path = str(tmp_path / "run.rst")
    with lbib.Solver(small_case(32, 16, 16, 8, 8, 10.0)) as s:
        s.run(2)
        s.save(path)
    other = Case(36, 16, 16, [centred_sheet(36, 16, 16, 8, 8, 0.5, 10.0)])
    with lbib.Solver(other) as s:
        with pytest.raises(lbib.LbibError):
            s.load(path)
    with lbib.Solver(small_case(32, 16, 16, 8, 8, 10.0), "f16") as s:
        with pytest.raises(lbib.LbibError):
            s.load(path)
        with pytest.raises(lbib.LbibError):
            s.load(str(tmp_path / "missing.rst"))
