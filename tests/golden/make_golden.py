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
  steps with the correctly rounded cosine, for the bit-exact GPU check.

Usage:  python tests/golden/make_golden.py [small|c0|c0cr|all]
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
from cases import SMALL_CASES, c0_case  # noqa: E402

C0_STEPS = 1000
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


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("small", "all"):
        make_small()
    if what in ("c0cr", "all"):
        make_c0_cr()
    if what in ("c0", "all"):
        make_c0()
