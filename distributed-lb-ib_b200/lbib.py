"""Python binding of liblbib.so (include/lbib.h) for tests, tools and bench.py.

The solver runs on the GPU through the C ABI only; there is no CPU path.
Loading fails loudly when the library is missing or was built for another
architecture.  Field arrays are x-fastest (``idx = (z*ny + y)*nx + x``) and
returned shaped (nz, ny, nx); sheet records are the reference's Fibernode
(12 doubles: x y z, bend xyz, stretch xyz, elastic xyz), shaped (rows, cols, 12).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("LBIB_LIBRARY") or os.path.join(HERE, "liblbib.so")

COMPAT_BEND_X_BUG = 1
COMPAT_YWALL_CUBES_X = 2
COMPAT_INOUT_PTHREAD = 4
COMPAT_ALL = 7

PREC_F64, PREC_F32, PREC_F16, PREC_BF16, PREC_SHIFT_FLOW = 0, 1, 2, 3, 16
# population storage: FP64 (the drop-in), or deviations from the rest
# weights ("f32", "f16", "bf16") or from the inflow equilibrium ("...-flow")
PRECISIONS = {"f64": PREC_F64, "f32": PREC_F32, "f16": PREC_F16, "bf16": PREC_BF16,
              "f32-flow": PREC_F32 | PREC_SHIFT_FLOW, "f16-flow": PREC_F16 | PREC_SHIFT_FLOW,
              "bf16-flow": PREC_BF16 | PREC_SHIFT_FLOW}

DUMP_NONE = 0
DUMP_FIELDVIEW = 1
DUMP_BINARY = 2

STAGES = {"bending": 0, "stretching": 1, "elastic": 2, "spread": 3, "collide": 4, "stream": 5,
          "bounceback": 6, "moments": 7, "move": 8, "copy_inout": 9, "replace": 10}

EXPORTED = [
    "init_gv_constant", "gen_fluid_grid", "gen_fiber_sheet", "init_gv", "init_eqlbrmdistrfuncDF0",
    "init_df1", "init_df_inout", "do_thread", "compute_bendingforce", "compute_stretchingforce",
    "compute_elasticforce", "fiber_SpreadForce", "fluid_get_SpreadForce",
    "get_influentialdomain_fluid_grid_and_SpreadForce", "compute_eqlbrmdistrfuncDF1", "stream_distrfunc",
    "bounceback_rigidwalls", "compute_rho_and_u", "fluid_SpreadVelocity", "fiber_get_SpreadVelocity",
    "moveFiberSheet", "copy_inout_to_df2", "replace_old_DF", "periodicBC", "save_fiber_sub_grid",
    "save_fiber_sub_grid_binary", "save_fluid_sub_grid", "save_fluid_sub_grid_vel_use_fv",
    "save_fluid_sub_grid_cord_use_fv", "save_fiber_sub_grid_cord_ef_use_fv", "lbib_set_params",
    "lbib_set_compat", "lbib_last_error", "lbib_error_string", "lbib_clear_error", "lbib_sync_to_host",
    "lbib_free", "lbib_get_moments", "lbib_get_force", "lbib_get_df1", "lbib_get_sheet", "lbib_set_sheet",
    "lbib_run", "lbib_synchronize", "lbib_stream", "lbib_case_create", "lbib_case_free", "lbib_stage",
    "lbib_device_count", "lbib_kernel_launches", "lbib_profile_begin", "lbib_profile_end",
    "lbib_set_precision", "lbib_case_create_prec", "lbib_spread_force_noalloc", "lbib_conservation_sums",
    "lbib_kernel_variants", "lbib_set_kernel_variant", "lbib_autotune",
    "lbib_batch_create", "lbib_batch_last_error", "lbib_batch_free", "lbib_batch_run", "lbib_batch_synchronize",
    "lbib_batch_stream", "lbib_batch_cells", "lbib_batch_steps", "lbib_batch_kernel_launches", "lbib_batch_status",
    "lbib_batch_get_sheet", "lbib_batch_get_moments", "lbib_batch_get_df1", "lbib_batch_variants",
    "lbib_batch_set_variant", "lbib_batch_autotune",
    "lbib_mlp_create", "lbib_mlp_free", "lbib_mlp_param_count", "lbib_mlp_stream", "lbib_mlp_get_params",
    "lbib_mlp_set_params", "lbib_mlp_forward", "lbib_mlp_gradient", "lbib_mlp_train_step", "lbib_mlp_synchronize",
    "lbib_save_restart", "lbib_load_restart", "lbib_mlp_set_stream",
    "lbib_set_slab", "lbib_case_create_slab", "lbib_slab_buffers", "lbib_slab_step_fluid",
    "lbib_slab_step_moments", "lbib_slab_moments", "lbib_slab_step_move",
    "lbib_slab_storage", "lbib_slab_connect", "lbib_slab_step_fluid_direct", "lbib_slab_step_moments_direct",
    "lbib_slab_check", "lbib_peer_access", "lbib_ipc_handle", "lbib_ipc_open", "lbib_ipc_close",
]

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib: Optional[C.CDLL] = None


class LbibError(RuntimeError):
    pass


def build(quiet: bool = True) -> str:
    """Compile liblbib.so in place (nvcc, sm_100a)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise LbibError("liblbib build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])
    if not quiet:
        print(out.stdout)
    return LIB_PATH


def load() -> C.CDLL:
    """Load liblbib.so and declare the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LbibError(f"{LIB_PATH} is missing; build it with `make -C {HERE}`")
    lib = C.CDLL(LIB_PATH)
    lib.lbib_case_create.restype = C.c_void_p
    lib.lbib_case_create.argtypes = [C.c_int] * 5 + [_ip, _ip] + [_dp] * 5 + [C.c_double] * 4 + [C.c_int]
    lib.lbib_case_create_prec.restype = C.c_void_p
    lib.lbib_case_create_prec.argtypes = lib.lbib_case_create.argtypes + [C.c_int]
    lib.lbib_set_precision.argtypes = [C.c_void_p, C.c_int]
    lib.lbib_case_free.argtypes = [C.c_void_p]
    lib.lbib_case_free.restype = None
    lib.lbib_run.argtypes = [C.c_void_p, C.c_int]
    lib.lbib_stage.argtypes = [C.c_void_p, C.c_int]
    for n in ["lbib_get_moments"]:
        getattr(lib, n).argtypes = [C.c_void_p] + [_dp] * 4
    lib.lbib_get_force.argtypes = [C.c_void_p] + [_dp] * 3
    lib.lbib_get_df1.argtypes = [C.c_void_p, _dp]
    lib.lbib_conservation_sums.argtypes = [C.c_void_p, _dp]
    lib.lbib_save_restart.argtypes = [C.c_void_p, C.c_char_p]
    lib.lbib_load_restart.argtypes = [C.c_void_p, C.c_char_p]
    lib.lbib_kernel_variants.argtypes = [C.c_void_p]
    lib.lbib_set_kernel_variant.argtypes = [C.c_void_p, C.c_int]
    lib.lbib_autotune.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int]
    lib.lbib_get_sheet.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.lbib_set_sheet.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.lbib_synchronize.argtypes = [C.c_void_p]
    lib.lbib_stream.argtypes = [C.c_void_p]
    lib.lbib_stream.restype = C.c_void_p
    lib.lbib_last_error.restype = C.c_int
    lib.lbib_error_string.argtypes = [C.c_int]
    lib.lbib_error_string.restype = C.c_char_p
    lib.lbib_clear_error.restype = None
    lib.lbib_set_compat.argtypes = [C.c_void_p, C.c_int]
    lib.lbib_set_params.argtypes = [C.c_void_p] + [C.c_double] * 4
    lib.lbib_device_count.restype = C.c_int
    lib.lbib_kernel_launches.argtypes = [C.c_void_p]
    lib.lbib_kernel_launches.restype = C.c_long
    lib.lbib_profile_begin.argtypes = [C.c_void_p]
    lib.lbib_profile_end.argtypes = [C.c_void_p, _dp, C.POINTER(C.c_long)]
    for n in ["init_gv_constant", "init_gv", "init_eqlbrmdistrfuncDF0", "init_df1", "init_df_inout",
              "lbib_free"]:
        getattr(lib, n).argtypes = [C.c_void_p]
        getattr(lib, n).restype = None
    lib.lbib_sync_to_host.argtypes = [C.c_void_p]
    lib.do_thread.argtypes = [C.c_void_p]
    lib.do_thread.restype = C.c_void_p
    lib.lbib_batch_create.restype = C.c_void_p
    lib.lbib_batch_create.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int]
    lib.lbib_batch_free.argtypes = [C.c_void_p]
    lib.lbib_batch_free.restype = None
    for n in ["lbib_batch_run"]:
        getattr(lib, n).argtypes = [C.c_void_p, C.c_int]
    for n in ["lbib_batch_synchronize", "lbib_batch_variants"]:
        getattr(lib, n).argtypes = [C.c_void_p]
    for n in ["lbib_batch_cells", "lbib_batch_steps", "lbib_batch_kernel_launches"]:
        getattr(lib, n).argtypes = [C.c_void_p]
        getattr(lib, n).restype = C.c_long
    lib.lbib_batch_stream.argtypes = [C.c_void_p]
    lib.lbib_batch_stream.restype = C.c_void_p
    lib.lbib_batch_status.argtypes = [C.c_void_p, _ip, _ip]
    lib.lbib_batch_get_sheet.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.lbib_batch_get_moments.argtypes = [C.c_void_p, C.c_int] + [_dp] * 4
    lib.lbib_batch_get_df1.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.lbib_batch_set_variant.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.lbib_batch_autotune.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int, _ip]
    _fp = C.POINTER(C.c_float)
    lib.lbib_mlp_create.restype = C.c_void_p
    lib.lbib_mlp_create.argtypes = [C.c_int, _ip, C.c_int, C.c_ulonglong]
    lib.lbib_mlp_free.argtypes = [C.c_void_p]
    lib.lbib_mlp_free.restype = None
    lib.lbib_mlp_param_count.argtypes = [C.c_void_p]
    lib.lbib_mlp_param_count.restype = C.c_long
    lib.lbib_mlp_stream.argtypes = [C.c_void_p]
    lib.lbib_mlp_stream.restype = C.c_void_p
    lib.lbib_mlp_get_params.argtypes = [C.c_void_p, _fp]
    lib.lbib_mlp_set_params.argtypes = [C.c_void_p, _fp]
    lib.lbib_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    lib.lbib_mlp_gradient.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, _fp, _fp]
    lib.lbib_mlp_train_step.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, _fp]
    lib.lbib_mlp_synchronize.argtypes = [C.c_void_p]
    lib.lbib_mlp_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    _lib = lib
    return lib


def device_count() -> int:
    return load().lbib_device_count()


def _check(rc: int, what: str) -> None:
    if rc != 0:
        msg = load().lbib_error_string(rc).decode()
        load().lbib_clear_error()
        raise LbibError(f"{what}: {msg} ({rc})")


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class Solver:
    """One LBM-IB problem on the GPU, set up through the reference-named API.

    ``case`` is any object with ``nx, ny, nz, cube_size, tau, u_l, Ks_l, Kb_l,
    compat`` and ``sheets`` (each with ``rows, cols, width, height, x0, y0,
    z0``), in the reference's internal axes (x = flow direction).
    ``precision`` (a key of PRECISIONS) selects the population storage;
    "f64" is the drop-in path.
    """

    def __init__(self, case, precision: str = "f64"):
        lib = load()
        self.lib = lib
        self.case = case
        sh: Sequence = case.sheets
        k = len(sh)
        ia = lambda v: (C.c_int * k)(*v)
        da = lambda v: (C.c_double * k)(*v)
        lib.lbib_clear_error()
        if precision not in PRECISIONS:
            raise LbibError(f"unknown precision {precision!r}")
        self.precision = precision
        self.gv = lib.lbib_case_create_prec(
            case.nx, case.ny, case.nz, case.cube_size, k,
            ia([s.rows for s in sh]), ia([s.cols for s in sh]),
            da([s.width for s in sh]), da([s.height for s in sh]),
            da([s.x0 for s in sh]), da([s.y0 for s in sh]), da([s.z0 for s in sh]),
            case.tau, case.u_l, case.Ks_l, case.Kb_l, case.compat, PRECISIONS[precision])
        if not self.gv:
            rc = lib.lbib_last_error()
            lib.lbib_clear_error()
            raise LbibError(f"lbib_case_create failed: {lib.lbib_error_string(rc).decode()} ({rc})")
        self.N = case.nx * case.ny * case.nz

    def close(self) -> None:
        if getattr(self, "gv", None):
            self.lib.lbib_case_free(self.gv)
            self.gv = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def run(self, nsteps: int) -> None:
        _check(self.lib.lbib_run(self.gv, nsteps), "lbib_run")

    def stage(self, name: str) -> None:
        _check(self.lib.lbib_stage(self.gv, STAGES[name]), "lbib_stage " + name)

    def synchronize(self) -> None:
        _check(self.lib.lbib_synchronize(self.gv), "lbib_synchronize")

    @property
    def stream(self) -> int:
        return self.lib.lbib_stream(self.gv) or 0

    @property
    def kernel_launches(self) -> int:
        return self.lib.lbib_kernel_launches(self.gv)

    def profile_begin(self) -> None:
        _check(self.lib.lbib_profile_begin(self.gv), "lbib_profile_begin")

    def profile_end(self):
        """Summed ms per stage (forces, spread, fluid, moments, move), steps."""
        ms = np.zeros(5)
        n = C.c_long(0)
        _check(self.lib.lbib_profile_end(self.gv, _ptr(ms), C.byref(n)), "lbib_profile_end")
        return dict(zip(["forces", "spread", "fluid", "moments", "move"], ms.tolist())), n.value

    def moments(self, out=None):
        """rho, ux, uy, uz as (nz, ny, nx) arrays; `out` (four C-contiguous
        float64 arrays of N values) is filled in place when given."""
        c = self.case
        if out is None:
            a = [np.empty(self.N) for _ in range(4)]
        else:
            a = list(out)
            if len(a) != 4 or any(x.dtype != np.float64 or x.size != self.N or not x.flags.c_contiguous for x in a):
                raise LbibError("moments(out=...): four C-contiguous float64 arrays of nx*ny*nz values")
        _check(self.lib.lbib_get_moments(self.gv, *[_ptr(x) for x in a]), "lbib_get_moments")
        return [x.reshape(c.nz, c.ny, c.nx) for x in a]

    def force(self):
        c = self.case
        a = [np.empty(self.N) for _ in range(3)]
        _check(self.lib.lbib_get_force(self.gv, *[_ptr(x) for x in a]), "lbib_get_force")
        return [x.reshape(c.nz, c.ny, c.nx) for x in a]

    def df1(self) -> np.ndarray:
        c = self.case
        a = np.empty(19 * self.N)
        _check(self.lib.lbib_get_df1(self.gv, _ptr(a)), "lbib_get_df1")
        return a.reshape(19, c.nz, c.ny, c.nx)

    def variants(self) -> int:
        n = self.lib.lbib_kernel_variants(self.gv)
        _check(min(n, 0), "lbib_kernel_variants")
        return n

    def set_variant(self, v: int) -> None:
        _check(self.lib.lbib_set_kernel_variant(self.gv, v), "lbib_set_kernel_variant")

    def autotune(self, steps: int = 8):
        """Pick the fastest fluid-kernel variant (before the first step).
        Returns (chosen variant, ms per step of each variant)."""
        ms = np.zeros(max(self.variants(), 1))
        best = self.lib.lbib_autotune(self.gv, steps, _ptr(ms), len(ms))
        _check(min(best, 0), "lbib_autotune")
        return best, ms.tolist()

    def save(self, path: str) -> None:
        """Restart file of the current state (lbib_save_restart)."""
        _check(self.lib.lbib_save_restart(self.gv, os.fsencode(path)), "lbib_save_restart")

    def load(self, path: str) -> None:
        _check(self.lib.lbib_load_restart(self.gv, os.fsencode(path)), "lbib_load_restart")

    def conservation(self) -> np.ndarray:
        """[mass, x, y, z momentum] of the populations, FP64 fixed-order sums."""
        a = np.empty(4)
        _check(self.lib.lbib_conservation_sums(self.gv, _ptr(a)), "lbib_conservation_sums")
        return a

    def sheet(self, k: int = 0) -> np.ndarray:
        s = self.case.sheets[k]
        a = np.empty(s.rows * s.cols * 12)
        _check(self.lib.lbib_get_sheet(self.gv, k, _ptr(a)), "lbib_get_sheet")
        return a.reshape(s.rows, s.cols, 12)

    def set_sheet(self, k: int, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        _check(self.lib.lbib_set_sheet(self.gv, k, _ptr(a)), "lbib_set_sheet")


class Problem(C.Structure):
    """One problem of a batch (lbib_problem)."""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("tau", C.c_double), ("u_l", C.c_double), ("Ks_l", C.c_double), ("Kb_l", C.c_double),
                ("rows", C.c_int), ("cols", C.c_int),
                ("width", C.c_double), ("height", C.c_double), ("x0", C.c_double), ("y0", C.c_double),
                ("z0", C.c_double), ("pinned", C.c_int)]

    @classmethod
    def from_case(cls, case):
        """From a one-sheet case object (the Solver's ``case``)."""
        s = case.sheets[0]
        return cls(case.nx, case.ny, case.nz, case.tau, case.u_l, case.Ks_l, case.Kb_l,
                   s.rows, s.cols, s.width, s.height, s.x0, s.y0, s.z0, int(getattr(case, "pinned", 0)))


class Batch:
    """Many independent one-sheet problems advanced together on the GPU
    (lbib_batch_*): one launch per stage for the whole batch, the step
    replayed as a CUDA graph."""

    def __init__(self, problems, precision: str = "f64", compat: int = COMPAT_ALL):
        lib = load()
        self.lib = lib
        if precision not in PRECISIONS:
            raise LbibError(f"unknown precision {precision!r}")
        self.problems = [p if isinstance(p, Problem) else Problem.from_case(p) for p in problems]
        arr = (Problem * len(self.problems))(*self.problems)
        self.h = lib.lbib_batch_create(len(self.problems), C.cast(arr, C.c_void_p), PRECISIONS[precision], compat)
        if not self.h:
            rc = lib.lbib_batch_last_error()
            raise LbibError(f"lbib_batch_create failed: {lib.lbib_error_string(rc).decode()} ({rc})")
        self.precision = precision

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.lbib_batch_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __len__(self):
        return len(self.problems)

    def run(self, nsteps: int) -> None:
        _check(self.lib.lbib_batch_run(self.h, nsteps), "lbib_batch_run")

    def synchronize(self) -> None:
        _check(self.lib.lbib_batch_synchronize(self.h), "lbib_batch_synchronize")

    @property
    def stream(self) -> int:
        return self.lib.lbib_batch_stream(self.h) or 0

    @property
    def cells(self) -> int:
        return self.lib.lbib_batch_cells(self.h)

    @property
    def steps(self) -> int:
        return self.lib.lbib_batch_steps(self.h)

    @property
    def kernel_launches(self) -> int:
        return self.lib.lbib_batch_kernel_launches(self.h)

    def status(self):
        """(codes, failed_step) per problem: 0 or LBIB_E_STENCIL (-3)."""
        n = len(self.problems)
        codes, steps = np.zeros(n, dtype=np.int32), np.zeros(n, dtype=np.int32)
        rc = self.lib.lbib_batch_status(self.h, codes.ctypes.data_as(_ip), steps.ctypes.data_as(_ip))
        _check(min(rc, 0), "lbib_batch_status")
        return codes, steps

    def sheet(self, k: int) -> np.ndarray:
        p = self.problems[k]
        a = np.empty(p.rows * p.cols * 12)
        _check(self.lib.lbib_batch_get_sheet(self.h, k, _ptr(a)), "lbib_batch_get_sheet")
        return a.reshape(p.rows, p.cols, 12)

    def moments(self, k: int):
        p = self.problems[k]
        n = p.nx * p.ny * p.nz
        a = [np.empty(n) for _ in range(4)]
        _check(self.lib.lbib_batch_get_moments(self.h, k, *[_ptr(x) for x in a]), "lbib_batch_get_moments")
        return [x.reshape(p.nz, p.ny, p.nx) for x in a]

    def df1(self, k: int) -> np.ndarray:
        p = self.problems[k]
        a = np.empty(19 * p.nx * p.ny * p.nz)
        _check(self.lib.lbib_batch_get_df1(self.h, k, _ptr(a)), "lbib_batch_get_df1")
        return a.reshape(19, p.nz, p.ny, p.nx)

    def variants(self) -> int:
        return self.lib.lbib_batch_variants(self.h)

    def set_variant(self, v: int, k: int = -1) -> None:
        _check(self.lib.lbib_batch_set_variant(self.h, k, v), "lbib_batch_set_variant")

    def autotune(self, steps: int = 6):
        """Pick a word-kernel variant per size class; returns (class of each
        problem, ms per step [class][variant])."""
        nv = self.variants()
        cls = np.zeros(len(self.problems), dtype=np.int32)
        ms = np.zeros(len(self.problems) * nv)
        n = self.lib.lbib_batch_autotune(self.h, steps, _ptr(ms), len(ms), cls.ctypes.data_as(_ip))
        _check(min(n, 0), "lbib_batch_autotune")
        return cls, ms[: n * nv].reshape(n, nv)


class MLP:
    """The GPU MLP of the sweep surrogate (lbib_mlp_*).  Arrays passed to
    forward / gradient / train_step are CUDA tensors (float32, contiguous,
    [batch, width]); torch only provides the device memory, and the MLP runs
    on the torch stream current at construction."""

    def __init__(self, widths, max_batch: int = 1024, seed: int = 0):
        lib = load()
        self.lib = lib
        self.widths = list(widths)
        w = (C.c_int * len(widths))(*widths)
        self.h = lib.lbib_mlp_create(len(widths) - 1, w, max_batch, seed)
        if not self.h:
            raise LbibError("lbib_mlp_create failed")
        self.max_batch = max_batch
        # run on torch's current stream: the batches torch gathers are then
        # ready before the MLP reads them, and not recycled while it does
        import torch
        _check(lib.lbib_mlp_set_stream(self.h, C.c_void_p(torch.cuda.current_stream().cuda_stream)),
               "lbib_mlp_set_stream")

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.lbib_mlp_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def nparams(self) -> int:
        return self.lib.lbib_mlp_param_count(self.h)

    def params(self) -> np.ndarray:
        a = np.empty(self.nparams, dtype=np.float32)
        _check(self.lib.lbib_mlp_get_params(self.h, a.ctypes.data_as(C.POINTER(C.c_float))), "lbib_mlp_get_params")
        return a

    def set_params(self, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float32)
        assert a.size == self.nparams
        _check(self.lib.lbib_mlp_set_params(self.h, a.ctypes.data_as(C.POINTER(C.c_float))), "lbib_mlp_set_params")

    @staticmethod
    def _dev(t, width):
        assert t.is_cuda and t.dtype.is_floating_point and t.is_contiguous() and t.shape[-1] == width
        return C.c_void_p(t.data_ptr())

    def forward(self, X):
        import torch
        Y = torch.empty((X.shape[0], self.widths[-1]), dtype=torch.float32, device=X.device)
        _check(self.lib.lbib_mlp_forward(self.h, self._dev(X, self.widths[0]), X.shape[0], self._dev(Y, self.widths[-1])),
               "lbib_mlp_forward")
        return Y

    def gradient(self, X, T):
        g = np.empty(self.nparams, dtype=np.float32)
        loss = C.c_float(0.0)
        _check(self.lib.lbib_mlp_gradient(self.h, self._dev(X, self.widths[0]), self._dev(T, self.widths[-1]),
                                          X.shape[0], g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)),
               "lbib_mlp_gradient")
        return g, loss.value

    def train_step(self, X, T, lr: float, want_loss: bool = False):
        loss = C.c_float(0.0)
        _check(self.lib.lbib_mlp_train_step(self.h, self._dev(X, self.widths[0]), self._dev(T, self.widths[-1]),
                                            X.shape[0], lr, C.byref(loss) if want_loss else None),
               "lbib_mlp_train_step")
        return loss.value if want_loss else None

    def synchronize(self) -> None:
        _check(self.lib.lbib_mlp_synchronize(self.h), "lbib_mlp_synchronize")
