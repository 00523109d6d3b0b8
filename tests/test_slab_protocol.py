"""The x-slab exchange rules on the CPU: a numpy model of the AA-pattern
D3Q19 step (the library's access rules: a link whose source is outside I
reads the cell's own slot, an odd-step push whose target is outside I goes to
the cell's own opposite slot) with a local stand-in for the collision, run on
the whole grid and on slabs that exchange exactly what csrc/lbib_slab.cu
exchanges -- after an even step the 5 populations with c_x pointing at the
neighbour into its ghost column (fill), after an odd step the ghost-bound
pushes back into the neighbour's column (flush), only rows where both ends of
the link lie in I.  The slabs must reproduce the whole grid slot for slot."""
import numpy as np
import pytest

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1])
CY = np.array([0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, -1, 1, 1, -1])
CZ = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0])
OPP = np.array([0] + [q + 1 if q % 2 else q - 1 for q in range(1, 19)])
PLUS = [q for q in range(19) if CX[q] == 1]      # the slots of lbib_slab.cu's face_q<+1>
MINUS = [q for q in range(19) if CX[q] == -1]


def test_tables():
    for q in range(19):
        assert (CX[OPP[q]], CY[OPP[q]], CZ[OPP[q]]) == (-CX[q], -CY[q], -CZ[q])
    assert PLUS == [1, 7, 9, 15, 17] and MINUS == [2, 8, 10, 16, 18]


class Grid:
    """Populations f[q, z, y, col] of global columns [x0, x0 + width)."""

    def __init__(self, nx, ny, nz, x0, width):
        self.nx, self.ny, self.nz, self.x0 = nx, ny, nz, x0
        self.f = np.zeros((19, nz, ny, width))

    def inI(self, x, y, z):
        return 2 <= x <= self.nx - 3 and 2 <= y <= self.ny - 3 and 2 <= z <= self.nz - 3

    def get(self, q, x, y, z):
        return self.f[q, z, y, x - self.x0]

    def put(self, q, x, y, z, v):
        self.f[q, z, y, x - self.x0] = v


def collide(f, x, y, z):
    """Any local map will do: the test compares two schedules of the same
    local arithmetic."""
    rho = f.sum()
    return f * (1.0 - 0.01 * (np.arange(19) % 5)) + 1e-3 * rho + 1e-4 * (x + 3 * y + 7 * z)


def step(g, par, xs):
    """One AA step of the cells of I with global x in xs (reads all, then
    writes all, as the kernel's cells do: every slot has one owner)."""
    out = []
    for z in range(2, g.nz - 2):
        for y in range(2, g.ny - 2):
            for x in xs:
                f = np.empty(19)
                for q in range(19):
                    if par == 0:
                        f[q] = g.get(q, x, y, z)
                    else:
                        xs_, ys, zs = x - CX[q], y - CY[q], z - CZ[q]
                        f[q] = g.get(OPP[q], xs_, ys, zs) if g.inI(xs_, ys, zs) else g.get(q, x, y, z)
                out.append((x, y, z, collide(f, x, y, z)))
    for x, y, z, f in out:
        for q in range(19):
            if par == 0:
                g.put(OPP[q], x, y, z, f[q])
            else:
                xt, yt, zt = x + CX[q], y + CY[q], z + CZ[q]
                if g.inI(xt, yt, zt):
                    g.put(q, xt, yt, zt, f[q])
                else:
                    g.put(OPP[q], x, y, z, f[q])


def rows_crossing(g, q):
    """(y, z) rows where a link of direction q crosses the face: the row and
    its source row both in I (lbib_halo_copy's unpack filter)."""
    for z in range(g.nz):
        for y in range(g.ny):
            ys, zs = y - CY[q], z - CZ[q]
            if 2 <= y <= g.ny - 3 and 2 <= z <= g.nz - 3 and 2 <= ys <= g.ny - 3 and 2 <= zs <= g.nz - 3:
                yield y, z


def copy_face(src, dst, xsrc, xdst, qs):
    for q in qs:
        for y, z in rows_crossing(dst, q):
            dst.put(q, xdst, y, z, src.get(q, xsrc, y, z))


def exchange(slabs, bounds, par):
    """lbdev_slab_pack + transport + lbdev_slab_unpack for every face."""
    for k in range(len(slabs) - 1):
        a, b = slabs[k], slabs[k + 1]
        X = bounds[k][1]                      # a owns [.., X), b owns [X, ..)
        if par == 0:                          # fill both ghosts
            copy_face(a, b, X - 1, X - 1, MINUS)
            copy_face(b, a, X, X, PLUS)
        else:                                 # flush both ghosts back
            copy_face(b, a, X - 1, X - 1, MINUS)
            copy_face(a, b, X, X, PLUS)


@pytest.mark.parametrize("bounds", [[(0, 8), (8, 16)], [(0, 4), (4, 12), (12, 16)]])
def test_slabs_reproduce_the_whole_grid(bounds):
    nx, ny, nz, steps = 16, 8, 8, 5
    rng = np.random.default_rng(0)
    whole = Grid(nx, ny, nz, 0, nx)
    whole.f[:] = rng.random(whole.f.shape)
    slabs = []
    for lo, hi in bounds:
        s = Grid(nx, ny, nz, lo - 2, hi - lo + 4)
        for x in range(max(lo - 2, 0), min(hi + 2, nx)):
            s.f[:, :, :, x - s.x0] = whole.f[:, :, :, x]
        slabs.append(s)
    I_x = range(2, nx - 2)
    for t in range(steps):
        par = t % 2
        step(whole, par, I_x)
        for s, (lo, hi) in zip(slabs, bounds):
            step(s, par, [x for x in I_x if lo <= x < hi])
        exchange(slabs, bounds, par)
        for s, (lo, hi) in zip(slabs, bounds):
            for x in range(lo, hi):
                if 2 <= x <= nx - 3:
                    np.testing.assert_array_equal(s.f[:, 2:nz - 2, 2:ny - 2, x - s.x0],
                                                  whole.f[:, 2:nz - 2, 2:ny - 2, x], err_msg=f"t={t} x={x}")


def test_without_the_row_filter_the_flush_clobbers_wall_rows():
    """The rule the filter encodes: at a wall row the receiving slab's cell
    writes the slot itself (bounce-back), so copying every row back breaks
    the result (the bug the GPU bit-comparison found first)."""
    nx, ny, nz = 16, 8, 8
    bounds = [(0, 8), (8, 16)]
    rng = np.random.default_rng(1)
    whole = Grid(nx, ny, nz, 0, nx)
    whole.f[:] = rng.random(whole.f.shape)
    slabs = []
    for lo, hi in bounds:
        s = Grid(nx, ny, nz, lo - 2, hi - lo + 4)
        for x in range(max(lo - 2, 0), min(hi + 2, nx)):
            s.f[:, :, :, x - s.x0] = whole.f[:, :, :, x]
        slabs.append(s)
    I_x = range(2, nx - 2)
    for t in range(2):
        step(whole, t, I_x)
        for s, (lo, hi) in zip(slabs, bounds):
            step(s, t, [x for x in I_x if lo <= x < hi])
        a, b = slabs
        if t == 0:
            exchange(slabs, bounds, 0)
        else:                                     # flush every row, unfiltered
            for q in MINUS:
                a.f[q, :, :, 7 - a.x0] = b.f[q, :, :, 7 - b.x0]
            for q in PLUS:
                b.f[q, :, :, 8 - b.x0] = a.f[q, :, :, 8 - a.x0]
    same = np.array_equal(slabs[0].f[:, 2:nz - 2, 2:ny - 2, 7 - slabs[0].x0], whole.f[:, 2:nz - 2, 2:ny - 2, 7])
    assert not same
