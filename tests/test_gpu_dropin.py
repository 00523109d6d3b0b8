"""The drop-in on the GPU: a host program written like the reference's
mpi/main.c (tests/c/drop_in_main.c), linked against liblbib.so, runs the
steps through do_thread; its results and its dump files are checked against
the oracle and against the reference's own output files."""
import os
import subprocess

import numpy as np
import pytest

import pyoracle as P
from cases import small_case

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "distributed-lb-ib_b200")


@pytest.fixture(scope="module")
def drop_in(tmp_path_factory, lbib_built):
    exe = tmp_path_factory.mktemp("bin") / "drop_in_main"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    out = subprocess.run([cc, "-std=gnu11", "-O2", "-I" + os.path.join(ROOT, "include"),
                          os.path.join(ROOT, "tests", "c", "drop_in_main.c"), "-L" + PKG, "-llbib",
                          "-Wl,-rpath," + PKG, "-o", str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return exe


def _args(case, steps, dump):
    s = case.sheets[0]
    return ["-steps", str(steps), "-dump", str(dump), "-fluid_grid_xyz", str(case.nx), str(case.ny), str(case.nz),
            "-cube_size", str(case.cube_size), "-num_fibersht", "1", "-fibersht_width_height", repr(s.width),
            repr(s.height), "-fibersht_row_clmn", str(s.rows), str(s.cols), "-fibersht_xyz_0", repr(s.x0),
            repr(s.y0), repr(s.z0), "-params", repr(case.tau), repr(case.u_l), repr(case.Ks_l), repr(case.Kb_l)]


def test_drop_in_program_matches_oracle(gpu, oracle_built, drop_in, tmp_path):
    case = small_case(24, 12, 12, 6, 6, 8.0)
    out = tmp_path / "state.bin"
    r = subprocess.run([str(drop_in)] + _args(case, 12, 1000) + ["-out", str(out)], capture_output=True,
                       text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "time 13"
    raw = np.fromfile(out, dtype=np.float64)
    S = case.sheets[0].rows * case.sheets[0].cols
    sheet = raw[:S * 12].reshape(case.sheets[0].rows, case.sheets[0].cols, 12)
    fields = raw[S * 12:].reshape(4, case.nz, case.ny, case.nx)
    o = P.Oracle(case, cr_cos=True)
    o.run(12)
    np.testing.assert_array_equal(sheet, o.sheet())
    for a, b in zip(fields, o.moments()):
        np.testing.assert_array_equal(a, b)


@pytest.mark.skipif(not P.reference_available(), reason="oracle/_ref not built")
def test_fieldview_files_match_reference_bytes(gpu, oracle_built, drop_in, tmp_path):
    """The reference always writes its FieldView files at time 1
    (cube_pthread/lbm_ib.c:3100-3112, 3503-3538); with -fv the drop-in writes
    the same files, byte for byte.  The one exception is the velocity file:
    the reference's writer indexes cubes with num_cubes_y and num_cubes_z
    left uninitialised (lbm_ib.c:445, used at :466), so its content is
    undefined; it is checked against the velocity field it names, formatted
    the same way ("%f," over z, y, x; u, then v, then w)."""
    case = small_case(24, 12, 12, 6, 6, 8.0)
    ref_dir = tmp_path / "ref"
    gpu_dir = tmp_path / "gpu"
    ref_dir.mkdir()
    gpu_dir.mkdir()
    ref = P.Reference(case, workdir=str(ref_dir))
    ref.run(1)
    r = subprocess.run([str(drop_in)] + _args(case, 1, 1000) + ["-fv"], capture_output=True, text=True,
                       cwd=gpu_dir)
    assert r.returncode == 0, r.stderr
    for n in ["FV_nameFluid.nam", "FV_nameFiber.nam", "FV_gridFluid.xyz", "FV_gridFiber1.xyz",
              "FV_fiber_elastic_force_1.f"]:
        assert (ref_dir / n).read_bytes() == (gpu_dir / n).read_bytes(), n
    o = P.Oracle(case, cr_cos=True)
    o.run(1)
    _, ux, uy, uz = o.moments()
    body = "".join("%f," % v for comp in (ux, uy, uz) for v in comp.ravel())
    want = f"{case.nx},{case.ny},{case.nz},3\n" + body
    assert (gpu_dir / "FV_fluid_vel_1.f").read_text() == want


def test_binary_fiber_dump(gpu, oracle_built, drop_in, tmp_path):
    """mpi/print_info.c:76-115 record layout: {int i, int j, Fibernode}
    (104 bytes), row-major, written every `dump` steps."""
    case = small_case(24, 12, 12, 6, 6, 8.0)
    r = subprocess.run([str(drop_in)] + _args(case, 4, 2) + ["-bin"], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    o = P.Oracle(case, cr_cos=True)
    rows, cols = case.sheets[0].rows, case.sheets[0].cols
    rec = np.dtype([("i", "<i4"), ("j", "<i4"), ("node", "<f8", (12,))])
    for step in (2, 4):
        o.run(2)
        data = np.fromfile(tmp_path / f"Fiber0_dump_step{step}.bin", dtype=rec)
        assert data.size == rows * cols and rec.itemsize == 104
        np.testing.assert_array_equal(data["i"], np.repeat(np.arange(rows), cols))
        np.testing.assert_array_equal(data["j"], np.tile(np.arange(cols), rows))
        np.testing.assert_array_equal(data["node"].reshape(rows, cols, 12), o.sheet())
