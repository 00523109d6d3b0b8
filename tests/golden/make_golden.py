"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own cube_pthread/lbm_ib.c (built into oracle/_ref by
oracle/Makefile from the reference checkout) serially, and stores what the
parity tests compare against:

* ``small_*.npz``  full rho, u fields and the full sheet records of small
  cases after a few steps (the oracle must reproduce them bit for bit; the
  CUDA path within the stated tolerance);
* ``c0_1000.npz``  the 128x64x64 / 52x52-sheet workload after 1000 steps:
  sheet records, rho/u at a fixed sample of 4096 cells and whole-field
  norms (the full fields would be 16 MB);
* ``c0_1000_cr.json``  sha256 of the oracle's fields after the same 1000
  steps with the correctly rounded cosine, for the bit-exact GPU check;
* ``c1_6.npz``  the 512x256x256 / 208x208-sheet workload (the benchmark's
  size) after 6 steps of the reference: every 4th sheet node's records
  (plus the last row and column), rho/u at 4096 random cells and at 4096
  cells of the box the sheet's delta stencils cover, and whole-field norms;
* ``c1_6_cr.json``  sha256 of the oracle's rho, u, sheet and interior
  populations after the same 6 steps with the correctly rounded cosine.

The c1 targets need ~28 GB (reference) and ~18 GB (oracle) of host memory.

Usage:  python tests/golden/make_golden.py [small|c0|c0cr|c1|c1cr|all]
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))

import pyoracle as P  # noqa: E402
from cases import SMALL_CASES, c0_case, c1_case  # noqa: E402

C0_STEPS = 1000
C1_STEPS = 6
SAMPLE_SEED = 1234
NSAMPLE = 4096


def c0_sample_index(case) -> np.ndarray:
    rng = np.random.default_rng(SAMPLE_SEED)
    return np.sort(rng.choice(case.ncells, size=NSAMPLE, replace=False))


def field_hash(fields) -> str:
    h = hashlib.sha256()
    for a in fields:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def make_small() -> None:
    for name, (case, steps) in SMALL_CASES.items():
        r = P.Reference(case)
        r.run(steps)
        rho, ux, uy, uz = r.moments()
        np.savez_compressed(os.path.join(HERE, f"small_{name}.npz"), rho=rho, ux=ux, uy=uy, uz=uz,
                            sheet=r.sheet(), steps=steps)
        print("wrote", name, steps, flush=True)


def make_c0() -> None:
    case = c0_case()
    r = P.Reference(case)
    t0 = time.time()
    r.run(C0_STEPS)
    rho, ux, uy, uz = r.moments()
    idx = c0_sample_index(case)
    np.savez_compressed(
        os.path.join(HERE, "c0_1000.npz"),
        sheet=r.sheet(), sample_idx=idx,
        rho=rho.ravel()[idx], ux=ux.ravel()[idx], uy=uy.ravel()[idx], uz=uz.ravel()[idx],
        norms=np.array([np.linalg.norm(rho), np.linalg.norm(ux), np.linalg.norm(uy), np.linalg.norm(uz)]),
        steps=C0_STEPS)
    print(f"wrote c0_1000 ({time.time() - t0:.0f} s)", flush=True)


def make_c0_cr() -> None:
    case = c0_case()
    P.Oracle.set_threads(os.cpu_count() or 1)
    o = P.Oracle(case, cr_cos=True)
    t0 = time.time()
    o.run(C0_STEPS)
    rho, ux, uy, uz = o.moments()
    sheet = o.sheet()
    out = {"steps": C0_STEPS, "moments_sha256": field_hash([rho, ux, uy, uz]),
           "sheet_sha256": field_hash([sheet]), "oracle": "liboracle_cr.so"}
    with open(os.path.join(HERE, "c0_1000_cr.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote c0_1000_cr.json ({time.time() - t0:.0f} s)", flush=True)


def c1_sample_index(case) -> np.ndarray:
    """4096 random cells of the grid and 4096 of the box x in [76, 84],
    y, z in the sheet's span +- 3 (where the spread force acts)."""
    rng = np.random.default_rng(SAMPLE_SEED)
    a = rng.choice(case.ncells, size=NSAMPLE, replace=False)
    s = case.sheets[0]
    xs = rng.integers(76, 85, NSAMPLE)
    ys = rng.integers(int(s.y0) - 3, int(s.y0 + s.height) + 4, NSAMPLE)
    zs = rng.integers(int(s.z0) - 3, int(s.z0 + s.width) + 4, NSAMPLE)
    b = (zs * case.ny + ys) * case.nx + xs
    return np.unique(np.concatenate([a, b]))


def c1_sheet_nodes(rows: int, cols: int):
    r = np.unique(np.r_[np.arange(0, rows, 4), rows - 1])
    c = np.unique(np.r_[np.arange(0, cols, 4), cols - 1])
    return r, c


def make_c1() -> None:
    case = c1_case()
    r = P.Reference(case)
    t0 = time.time()
    r.run(C1_STEPS)
    rho, ux, uy, uz = r.moments()
    idx = c1_sample_index(case)
    s = case.sheets[0]
    rr, cc = c1_sheet_nodes(s.rows, s.cols)
    sheet = r.sheet()
    np.savez_compressed(
        os.path.join(HERE, "c1_6.npz"),
        sheet_rows=rr, sheet_cols=cc, sheet=sheet[np.ix_(rr, cc)], sample_idx=idx,
        sheet_norm=np.linalg.norm(sheet[..., :3]),
        rho=rho.ravel()[idx], ux=ux.ravel()[idx], uy=uy.ravel()[idx], uz=uz.ravel()[idx],
        norms=np.array([np.linalg.norm(rho), np.linalg.norm(ux), np.linalg.norm(uy), np.linalg.norm(uz)]),
        steps=C1_STEPS)
    print(f"wrote c1_6 ({time.time() - t0:.0f} s)", flush=True)


def c1_interior_df_hash(df) -> str:
    """sha256 of the populations of the cells that collide, (q, z, y, x) order."""
    h = hashlib.sha256()
    nq, nz, ny, nx = df.shape
    for q in range(nq):
        h.update(np.ascontiguousarray(df[q, 2:nz - 2, 2:ny - 2, 2:nx - 2]).tobytes())
    return h.hexdigest()


def make_c1_cr() -> None:
    case = c1_case()
    P.Oracle.set_threads(os.cpu_count() or 1)
    o = P.Oracle(case, cr_cos=True)
    t0 = time.time()
    o.run(C1_STEPS)
    rho, ux, uy, uz = o.moments()
    out = {"steps": C1_STEPS, "moments_sha256": field_hash([rho, ux, uy, uz]),
           "sheet_sha256": field_hash([o.sheet()]), "oracle": "liboracle_cr.so"}
    del rho, ux, uy, uz
    out["df1_interior_sha256"] = c1_interior_df_hash(o.df(0))
    with open(os.path.join(HERE, "c1_6_cr.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote c1_6_cr.json ({time.time() - t0:.0f} s)", flush=True)


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("small", "all"):
        make_small()
    if what in ("c0cr", "all"):
        make_c0_cr()
    if what in ("c0", "all"):
        make_c0()
    if what in ("c1cr", "all"):
        make_c1_cr()
    if what in ("c1", "all"):
        make_c1()
