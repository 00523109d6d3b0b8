"""The drop-in boundary: liblbib.so loads without a GPU, exports every
function include/lbib.h declares, and a host program written like the
reference's mpi/main.c compiles and links against it."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import lbib
import pyoracle as P
from cases import small_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lbib.h")
PKG = os.path.join(ROOT, "distributed-lb-ib_b200")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("typedef",)))


def test_header_declares_reference_api():
    names = declared_functions()
    for n in ["init_gv_constant", "gen_fluid_grid", "gen_fiber_sheet", "init_gv", "init_eqlbrmdistrfuncDF0",
              "init_df1", "init_df_inout", "do_thread", "compute_eqlbrmdistrfuncDF1", "moveFiberSheet",
              "save_fiber_sub_grid_binary", "lbib_last_error"]:
        assert n in names


def test_library_exports_every_declared_symbol(lbib_built):
    lib = ctypes.CDLL(lbib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(lbib.EXPORTED) <= set(declared_functions())


def test_binding_loads_without_gpu(lbib_built):
    lib = lbib.load()
    assert lib.lbib_error_string(-3).decode().startswith("a fiber node")
    assert lbib.device_count() >= 0


def _build_drop_in(tmp_path):
    exe = tmp_path / "drop_in_main"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    out = subprocess.run([cc, "-std=gnu11", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"),
                          os.path.join(ROOT, "tests", "c", "drop_in_main.c"), "-L" + PKG, "-llbib",
                          "-Wl,-rpath," + PKG, "-o", str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return exe


def test_drop_in_host_setup_matches_oracle(lbib_built, oracle_built, tmp_path):
    """Host-only set-up through the reference-named API (no GPU calls)."""
    exe = _build_drop_in(tmp_path)
    case = small_case(24, 12, 12, 6, 6, 8.0)
    s = case.sheets[0]
    out = tmp_path / "host.txt"
    r = subprocess.run([str(exe), "-steps", "3", "-dump", "100", "-fluid_grid_xyz", "24", "12", "12",
                        "-cube_size", "4", "-num_fibersht", "1", "-fibersht_width_height", repr(s.width),
                        repr(s.height), "-fibersht_row_clmn", str(s.rows), str(s.cols), "-fibersht_xyz_0",
                        repr(s.x0), repr(s.y0), repr(s.z0), "-host_only", "-out", str(out)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = out.read_text().splitlines()
    assert lines[0] == "dt 1 time 1 ib 2 ie 21 jb 2 je 9 kb 2 ke 9"
    consts = dict(zip(lines[1].split()[0::2], map(float, lines[1].split()[1::2])))
    # mpi/init_gv.c:74-97 hard-coded physics
    assert consts["u_l"] == 0.001 and consts["tau"] == 0.5 * (6.0 * (0.001 * 20.0 / 150.0) + 1.0)
    assert consts["Kb_l"] == 0.005 * 1.0 * 0.001 * 0.001 * 20.0 ** 4
    assert lines[2] == "cubes 6 3 3"
    nodes = np.array([[float(v) for v in l.split()[4:]] for l in lines[3:]])
    # gen_fiber_sheet positions (before init_gv's shift) equal the oracle's minus u_l*dt
    o = P.Oracle(P.Case(24, 12, 12, case.sheets, u_l=0.0))
    np.testing.assert_array_equal(nodes, o.sheet()[..., :3].reshape(-1, 3))


def test_precision_arguments_checked_before_any_gpu_call(lbib_built):
    """Unknown storage precisions are refused on the host (no CUDA call)."""
    lib = lbib.load()
    one_i = (ctypes.c_int * 1)(4)
    one_d = (ctypes.c_double * 1)(1.0)
    lib.lbib_clear_error()
    for bad in (-1, 4, 16, 20, 99):
        gv = lib.lbib_case_create_prec(32, 16, 16, 4, 1, one_i, one_i, one_d, one_d, one_d, one_d, one_d,
                                       0.6, 0.01, 0.05, 0.005, P.COMPAT_ALL, bad)
        assert not gv
        assert lib.lbib_last_error() == -1
        lib.lbib_clear_error()
    assert lib.lbib_set_precision(None, lbib.PREC_F16) == -1
    lib.lbib_clear_error()
    assert lbib.PRECISIONS["f64"] == 0 and lbib.PRECISIONS["f16-flow"] == 18
    with pytest.raises(lbib.LbibError):
        lbib.Solver(small_case(), precision="f8")


def test_batch_arguments_checked_before_any_gpu_call(lbib_built):
    lib = lbib.load()
    good = lbib.Problem(32, 16, 16, 0.6, 0.01, 0.05, 0.005, 4, 4, 1.5, 1.5, 10.0, 7.0, 7.0, 0)
    for bad in [lbib.Problem(30, 16, 16, 0.6, 0.01, 0.05, 0.005, 4, 4, 1.5, 1.5, 10.0, 7.0, 7.0),   # not /4
                lbib.Problem(32, 16, 16, 0.5, 0.01, 0.05, 0.005, 4, 4, 1.5, 1.5, 10.0, 7.0, 7.0),   # tau
                lbib.Problem(32, 16, 16, 0.6, 0.01, 0.05, 0.005, 1, 4, 1.5, 1.5, 10.0, 7.0, 7.0)]:  # rows
        arr = (lbib.Problem * 2)(good, bad)
        assert not lib.lbib_batch_create(2, ctypes.cast(arr, ctypes.c_void_p), 0, 7)
        assert lib.lbib_batch_last_error() == -1
    arr = (lbib.Problem * 1)(good)
    for prec in (-1, 4, 16):
        assert not lib.lbib_batch_create(1, ctypes.cast(arr, ctypes.c_void_p), prec, 7)
    assert not lib.lbib_batch_create(0, None, 0, 7)
