"""ctypes bindings for the oracle -- TEST INFRASTRUCTURE ONLY.

Two CPU implementations of the reference time step live under oracle/:

* ``Oracle`` wraps liboracle.so, the C restatement (oracle/lbib_oracle.c);
* ``Reference`` wraps _ref/libref.so, the reference's own
  cube_pthread/lbm_ib.c compiled with the serial driver oracle/ref_harness.c.

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs use
this module, as the checker.  Field arrays are x-fastest,
``idx = (z*ny + y)*nx + x``, returned as numpy arrays shaped (nz, ny, nx).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
ORACLE_CR_SO = os.path.join(HERE, "liboracle_cr.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")

COMPAT_BEND_X_BUG = 1
COMPAT_YWALL_CUBES_X = 2
COMPAT_INOUT_PTHREAD = 4
COMPAT_ALL = 7

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


@dataclass
class Sheet:
    """One fiber sheet as the reference's -fibersht_* flags describe it."""
    rows: int
    cols: int
    width: float
    height: float
    x0: float
    y0: float
    z0: float


@dataclass
class Case:
    """A complete LBM-IB problem in the reference's internal axes (x = flow)."""
    nx: int
    ny: int
    nz: int
    sheets: List[Sheet]
    tau: float = 0.6
    u_l: float = 0.01
    Ks_l: float = 0.05
    Kb_l: float = 0.005
    cube_size: int = 4
    compat: int = COMPAT_ALL

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz


def build(quiet: bool = True) -> None:
    """Run oracle/Makefile (restatement always; _ref when the reference exists)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class _Base:
    lib: C.CDLL

    def _arr(self, n: int) -> np.ndarray:
        return np.empty(n, dtype=np.float64)


class Oracle(_Base):
    """The C restatement of the reference step (SoA, serial arithmetic order).

    ``cr_cos=False`` uses the C library's cosine in the delta kernel, exactly
    as the reference does; ``cr_cos=True`` uses the correctly rounded cosine
    of the CUDA path, for bit-for-bit comparisons with it.
    """

    _libs: dict = {}

    @classmethod
    def load(cls, cr_cos: bool = False) -> C.CDLL:
        path = ORACLE_CR_SO if cr_cos else ORACLE_SO
        if path not in cls._libs:
            if not os.path.exists(path):
                build()
            lib = C.CDLL(path)
            lib.orc_create.restype = C.c_void_p
            lib.orc_create.argtypes = [C.c_int] * 5 + [_ip, _ip] + [_dp] * 5 + [C.c_double] * 4 + [C.c_int]
            for name in ["orc_bending", "orc_stretching", "orc_elastic", "orc_collide", "orc_stream",
                         "orc_bounceback", "orc_moments", "orc_copy_inout", "orc_replace", "orc_free"]:
                getattr(lib, name).argtypes = [C.c_void_p]
                getattr(lib, name).restype = None
            for name in ["orc_spread", "orc_move", "orc_step", "orc_time"]:
                getattr(lib, name).argtypes = [C.c_void_p]
                getattr(lib, name).restype = C.c_int
            lib.orc_run.argtypes = [C.c_void_p, C.c_int]
            lib.orc_run.restype = C.c_int
            lib.orc_get_moments.argtypes = [C.c_void_p] + [_dp] * 4
            lib.orc_set_moments.argtypes = [C.c_void_p] + [_dp] * 4
            lib.orc_get_force.argtypes = [C.c_void_p] + [_dp] * 3
            lib.orc_set_force.argtypes = [C.c_void_p] + [_dp] * 3
            lib.orc_get_df.argtypes = [C.c_void_p, C.c_int, _dp]
            lib.orc_set_df.argtypes = [C.c_void_p, C.c_int, _dp]
            lib.orc_get_inout.argtypes = [C.c_void_p, C.c_int, _dp]
            lib.orc_get_sheet.argtypes = [C.c_void_p, C.c_int, _dp]
            lib.orc_set_sheet.argtypes = [C.c_void_p, C.c_int, _dp]
            lib.orc_set_threads.argtypes = [C.c_int]
            cls._libs[path] = lib
        return cls._libs[path]

    def __init__(self, case: Case, cr_cos: bool = False):
        self.lib = self.load(cr_cos)
        self.case = case
        k = len(case.sheets)
        ia = lambda v: (C.c_int * k)(*v)
        da = lambda v: (C.c_double * k)(*v)
        sh = case.sheets
        self.h = self.lib.orc_create(
            case.nx, case.ny, case.nz, case.cube_size, k,
            ia([s.rows for s in sh]), ia([s.cols for s in sh]),
            da([s.width for s in sh]), da([s.height for s in sh]),
            da([s.x0 for s in sh]), da([s.y0 for s in sh]), da([s.z0 for s in sh]),
            case.tau, case.u_l, case.Ks_l, case.Kb_l, case.compat)
        if not self.h:
            raise ValueError("oracle rejected the case (cube size / divisibility)")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_free(self.h)
            self.h = None

    @staticmethod
    def set_threads(n: int) -> None:
        Oracle.load(False).orc_set_threads(n)
        Oracle.load(True).orc_set_threads(n)

    def stage(self, name: str) -> int:
        r = getattr(self.lib, "orc_" + name)(self.h)
        return 0 if r is None else r

    def run(self, nsteps: int) -> None:
        if self.lib.orc_run(self.h, nsteps) != 0:
            raise RuntimeError("oracle: a fiber stencil left the fluid grid")

    @property
    def time(self) -> int:
        return self.lib.orc_time(self.h)

    def moments(self):
        c = self.case
        a = [self._arr(c.ncells) for _ in range(4)]
        self.lib.orc_get_moments(self.h, *[_ptr(x) for x in a])
        return [x.reshape(c.nz, c.ny, c.nx) for x in a]

    def set_moments(self, rho, ux, uy, uz) -> None:
        a = [np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (rho, ux, uy, uz)]
        self.lib.orc_set_moments(self.h, *[_ptr(x) for x in a])

    def force(self):
        c = self.case
        a = [self._arr(c.ncells) for _ in range(3)]
        self.lib.orc_get_force(self.h, *[_ptr(x) for x in a])
        return [x.reshape(c.nz, c.ny, c.nx) for x in a]

    def set_force(self, fx, fy, fz) -> None:
        a = [np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (fx, fy, fz)]
        self.lib.orc_set_force(self.h, *[_ptr(x) for x in a])

    def df(self, which: int = 0) -> np.ndarray:
        c = self.case
        a = self._arr(19 * c.ncells)
        self.lib.orc_get_df(self.h, which, _ptr(a))
        return a.reshape(19, c.nz, c.ny, c.nx)

    def set_df(self, which: int, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        self.lib.orc_set_df(self.h, which, _ptr(a))

    def inout(self, which: int) -> np.ndarray:
        c = self.case
        a = self._arr(19 * c.ny * c.nz)
        self.lib.orc_get_inout(self.h, which, _ptr(a))
        return a.reshape(19, c.ny, c.nz)

    def sheet(self, k: int = 0) -> np.ndarray:
        s = self.case.sheets[k]
        a = self._arr(s.rows * s.cols * 12)
        self.lib.orc_get_sheet(self.h, k, _ptr(a))
        return a.reshape(s.rows, s.cols, 12)

    def set_sheet(self, k: int, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        self.lib.orc_set_sheet(self.h, k, _ptr(a))


REF_STAGES = {"bending": 0, "stretching": 1, "elastic": 2, "spread": 3, "collide": 4, "stream": 5,
              "bounceback": 6, "moments": 7, "move": 8, "copy_inout": 9, "replace": 10, "tick": 11}


def reference_available() -> bool:
    return os.path.exists(REF_SO)


class Reference(_Base):
    """The reference's own cube_pthread/lbm_ib.c, driven serially (one sheet)."""

    _lib: Optional[C.CDLL] = None

    @classmethod
    def load(cls) -> C.CDLL:
        if cls._lib is None:
            if not os.path.exists(REF_SO):
                raise FileNotFoundError(REF_SO + " (build it with make -C oracle ref)")
            lib = C.CDLL(REF_SO)
            lib.ref_create.restype = C.c_void_p
            lib.ref_create.argtypes = [C.c_int] * 6 + [C.c_double] * 9
            lib.ref_run.argtypes = [C.c_void_p, C.c_int, C.c_char_p]
            lib.ref_run.restype = C.c_int
            lib.ref_run_threaded.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_char_p]
            lib.ref_run_threaded.restype = C.c_int
            lib.ref_call.argtypes = [C.c_void_p, C.c_int]
            lib.ref_call.restype = C.c_int
            lib.ref_time.argtypes = [C.c_void_p]
            lib.ref_time.restype = C.c_int
            for n in ["ref_get_moments", "ref_set_moments"]:
                getattr(lib, n).argtypes = [C.c_void_p] + [_dp] * 4
            for n in ["ref_get_force", "ref_set_force"]:
                getattr(lib, n).argtypes = [C.c_void_p] + [_dp] * 3
            lib.ref_get_df.argtypes = [C.c_void_p, C.c_int, _dp]
            lib.ref_set_df.argtypes = [C.c_void_p, C.c_int, _dp]
            lib.ref_get_inout.argtypes = [C.c_void_p, C.c_int, _dp]
            lib.ref_get_sheet.argtypes = [C.c_void_p, _dp]
            lib.ref_set_sheet.argtypes = [C.c_void_p, _dp]
            lib.ref_free.argtypes = [C.c_void_p]
            cls._lib = lib
        return cls._lib

    def __init__(self, case: Case, workdir: Optional[str] = None):
        if len(case.sheets) != 1:
            raise ValueError("the reference step handles sheets[0] only")
        if case.compat != COMPAT_ALL:
            raise ValueError("the reference has every compat behaviour built in")
        self.lib = self.load()
        self.case = case
        s = case.sheets[0]
        self.h = self.lib.ref_create(case.nx, case.ny, case.nz, case.cube_size, s.rows, s.cols,
                                     s.width, s.height, s.x0, s.y0, s.z0,
                                     case.tau, case.u_l, case.Ks_l, case.Kb_l)
        self._tmp = None
        if workdir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="lbib_ref_")
            workdir = self._tmp.name
        self.workdir = workdir

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_free(self.h)
            self.h = None

    def run(self, nsteps: int) -> None:
        if self.lib.ref_run(self.h, nsteps, self.workdir.encode()) != 0:
            raise RuntimeError("reference run failed")

    def run_threaded(self, nsteps: int, Q: int, R: int) -> None:
        r = self.lib.ref_run_threaded(self.h, nsteps, Q, R, self.workdir.encode())
        if r != 0:
            raise RuntimeError(f"reference threaded run failed ({r})")

    def stage(self, name: str) -> int:
        return self.lib.ref_call(self.h, REF_STAGES[name])

    @property
    def time(self) -> int:
        return self.lib.ref_time(self.h)

    def moments(self):
        c = self.case
        a = [self._arr(c.ncells) for _ in range(4)]
        self.lib.ref_get_moments(self.h, *[_ptr(x) for x in a])
        return [x.reshape(c.nz, c.ny, c.nx) for x in a]

    def set_moments(self, rho, ux, uy, uz) -> None:
        a = [np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (rho, ux, uy, uz)]
        self.lib.ref_set_moments(self.h, *[_ptr(x) for x in a])

    def force(self):
        c = self.case
        a = [self._arr(c.ncells) for _ in range(3)]
        self.lib.ref_get_force(self.h, *[_ptr(x) for x in a])
        return [x.reshape(c.nz, c.ny, c.nx) for x in a]

    def set_force(self, fx, fy, fz) -> None:
        a = [np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (fx, fy, fz)]
        self.lib.ref_set_force(self.h, *[_ptr(x) for x in a])

    def df(self, which: int = 0) -> np.ndarray:
        c = self.case
        a = self._arr(19 * c.ncells)
        self.lib.ref_get_df(self.h, which, _ptr(a))
        return a.reshape(19, c.nz, c.ny, c.nx)

    def set_df(self, which: int, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        self.lib.ref_set_df(self.h, which, _ptr(a))

    def inout(self, which: int) -> np.ndarray:
        c = self.case
        a = self._arr(19 * c.ny * c.nz)
        self.lib.ref_get_inout(self.h, which, _ptr(a))
        return a.reshape(19, c.ny, c.nz)

    def sheet(self, k: int = 0) -> np.ndarray:
        s = self.case.sheets[0]
        a = self._arr(s.rows * s.cols * 12)
        self.lib.ref_get_sheet(self.h, _ptr(a))
        return a.reshape(s.rows, s.cols, 12)

    def set_sheet(self, k: int, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        self.lib.ref_set_sheet(self.h, _ptr(a))


def centred_sheet(nx: int, ny: int, nz: int, rows: int, cols: int, spacing: float, x0: float) -> Sheet:
    """A rows x cols sheet at `spacing`, in the plane x = x0, centred in y and z."""
    w = spacing * (cols - 1)
    h = spacing * (rows - 1)
    return Sheet(rows=rows, cols=cols, width=w, height=h, x0=x0,
                 y0=(ny - 1) / 2.0 - h / 2.0, z0=(nz - 1) / 2.0 - w / 2.0)
