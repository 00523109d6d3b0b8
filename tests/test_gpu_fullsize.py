"""Size-independent properties at the headline size (512 x 256 x 256, one
208 x 208 sheet), where the oracle is too slow to run: the two-cell kernel
and the one-cell kernel give the same bits, two runs give the same bits,
and the grid cut into x-slabs gives the whole grid's bits (both exchanges).
Populations are compared through their FP64 fixed-order sums and the sheet
records (the sheet integrates the velocity field around it every step)."""
import numpy as np
import pytest

import lbib
import slabs
from cases import c1_case

pytestmark = pytest.mark.gpu
STEPS = 6     # both AA parities, three times


def _run(case, steps):
    with lbib.Solver(case) as s:
        s.run(steps)
        return s.sheet(), s.conservation()


@pytest.fixture(scope="module")
def whole():
    return _run(c1_case(), STEPS)


def test_c1_two_cell_and_one_cell_kernels_agree(gpu, whole, monkeypatch):
    monkeypatch.setenv("LBIB_FLUID_BULK", "0")
    sheet, sums = _run(c1_case(), STEPS)
    assert np.array_equal(sheet, whole[0])
    assert np.array_equal(sums, whole[1])
    assert np.abs(sheet[..., 0] - c1_case().sheets[0].x0).max() > 0.05     # the sheet moved


def test_c1_deterministic(gpu, whole):
    sheet, sums = _run(c1_case(), STEPS)
    assert np.array_equal(sheet, whole[0]) and np.array_equal(sums, whole[1])


@pytest.mark.parametrize("direct", [False, True])
def test_c1_slabs_equal_whole(gpu, whole, direct):
    # the sheet (x ~ 80) straddles the face at x = 80 of the first cut
    with slabs.LocalSlabs(c1_case(), bounds=[(0, 80), (80, 296), (296, 512)], direct=direct) as L:
        L.run(STEPS)
        assert np.array_equal(L.sheet(), whole[0])
