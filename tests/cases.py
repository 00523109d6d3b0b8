"""Parity-test cases, in the reference's internal axes (x = flow direction).

The workloads follow the benchmark definitions: D3Q19 with tau = 0.6,
inflow u_x = 0.01, Ks = 0.05, Kb = 0.005 and sheets at 0.5 node spacing
centred in y and z.  Small cases exercise the same code paths on grids the
oracle finishes in well under a second.
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))

from pyoracle import COMPAT_ALL, Case, Sheet, centred_sheet  # noqa: E402


def c0_case() -> Case:
    """128(x) x 64(y) x 64(z), one 52x52 sheet at x = 20 (the reference's own size)."""
    nx, ny, nz = 128, 64, 64
    return Case(nx, ny, nz, [centred_sheet(nx, ny, nz, 52, 52, 0.5, 20.0)])


def c1_case() -> Case:
    """512 x 256 x 256, one 208x208 sheet at x = 80."""
    nx, ny, nz = 512, 256, 256
    return Case(nx, ny, nz, [centred_sheet(nx, ny, nz, 208, 208, 0.5, 80.0)])


def small_case(nx=32, ny=16, nz=16, rows=8, cols=8, x0=10.0, **kw) -> Case:
    return Case(nx, ny, nz, [centred_sheet(nx, ny, nz, rows, cols, 0.5, x0)], **kw)


# name -> (case, steps); the golden fixtures store the reference's state after `steps`
SMALL_CASES = {
    # default physics, a sheet that bends and moves
    "base": (small_case(24, 12, 12, 6, 6, 8.0), 40),
    # num_cubes_x < num_cubes_z: the reference's loop-bound bugs are active
    "xltz": (small_case(12, 12, 24, 6, 6, 5.0), 25),
    # stiff sheet off-centre near a z wall, rows != cols
    "wall": (Case(32, 16, 16, [Sheet(8, 6, 2.5, 3.5, 9.0, 4.0, 3.5)], Ks_l=0.5, Kb_l=0.05), 30),
}
