"""The field getter's two read-back paths give the same bits.

lbib_get_moments writes page-locked (mapped) host arrays directly from the
moments kernel and stages pageable ones in device memory first; both must
return the same rho and u, before the first step and after steps of both
parities, in FP64 and in 16-bit storage."""
import numpy as np
import pytest
import torch

import lbib
from cases import small_case

pytestmark = pytest.mark.gpu


def _pinned(n):
    return [torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for _ in range(4)]


@pytest.mark.parametrize("steps", [0, 1, 4])
def test_moments_into_pinned_equal_pageable(gpu, steps):
    case = small_case(32, 16, 16, 8, 8, 10.0)
    with lbib.Solver(case) as s:
        s.run(steps)
        a = s.moments()
        out = _pinned(case.nx * case.ny * case.nz)
        for x in out:
            x.fill(np.nan)
        b = s.moments(out=out)
        for u, v in zip(a, b):
            assert np.array_equal(u.view(np.int64), v.view(np.int64))
        assert all(np.isfinite(x).all() for x in out)    # every cell written


def test_moments_into_pinned_low_precision(gpu):
    case = small_case(32, 16, 16, 8, 8, 10.0)
    with lbib.Solver(case, precision="f16-flow") as s:
        s.run(3)
        a = s.moments()
        b = s.moments(out=_pinned(case.nx * case.ny * case.nz))
        for u, v in zip(a, b):
            assert np.array_equal(u.view(np.int64), v.view(np.int64))
