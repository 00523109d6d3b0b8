"""The delta kernel's cosine.

The CUDA path evaluates 1 + cos(pi/2 r) with a correctly rounded double-double
cosine (distributed-lb-ib_b200/csrc/lbib_cos.h).  Checked here against a
60-digit decimal evaluation, including arguments where the C library's cosine
(which the reference calls) is 1 ulp off.
"""
import ctypes as C
import math
from decimal import Decimal, getcontext

import numpy as np
import pytest

import pyoracle as P

getcontext().prec = 60
PI_T = 3.14159265358979  # the reference's truncated PI, cube_pthread/lbm_ib.c:33


def cos_hp(x: float) -> Decimal:
    d = Decimal(x)
    s = Decimal(1)
    t = Decimal(1)
    n = 0
    while True:
        n += 2
        t = -t * d * d / ((n - 1) * n)
        if abs(t) < Decimal(10) ** -58:
            return s
        s += t


def is_correctly_rounded(x: float, v: float) -> bool:
    e = cos_hp(x)
    err = abs(Decimal(v) - e)
    return all(err <= abs(Decimal(math.nextafter(v, d)) - e) for d in (math.inf, -math.inf))


def _cos_fns():
    cr = P.Oracle.load(cr_cos=True)
    lm = P.Oracle.load(cr_cos=False)
    for lib in (cr, lm):
        lib.orc_cos.restype = C.c_double
        lib.orc_cos.argtypes = [C.c_double]
    return cr.orc_cos, lm.orc_cos


def delta_args(n: int, seed: int) -> np.ndarray:
    """Arguments as the delta kernel forms them: pi/2 * (gi - X)."""
    rng = np.random.default_rng(seed)
    X = rng.uniform(2.0, 200.0, n)
    gi = np.floor(X - 2) + 1 + rng.integers(0, 4, n)
    return (PI_T / 2.0) * (gi - X)


def test_cr_cosine_is_correctly_rounded(oracle_built):
    cr, lm = _cos_fns()
    xs = list(delta_args(1500, 5)) + [0.0, 1e-9, -1e-9, 0.5, 1.0, PI_T / 2, -PI_T / 2, PI_T, -PI_T,
                                      math.pi / 2, math.pi / 4, 3 * math.pi / 4, 2.0, -3.1]
    # arguments where glibc's cos is 1 ulp off (found by scanning)
    xs += [1.2231614256588297, 0.47938056872090196, -2.1501599567293868, 1.7759313193883071]
    bad = [x for x in xs if not is_correctly_rounded(x, cr(x))]
    assert not bad, bad[:5]


def test_libm_cosine_differs_on_a_small_fraction(oracle_built):
    """Why the CUDA path is compared with the reference by tolerance: the C
    library's cosine mis-rounds a small fraction of these arguments."""
    cr, lm = _cos_fns()
    xs = delta_args(100000, 9)
    diff = sum(cr(float(x)) != lm(float(x)) for x in xs)
    assert 0 < diff < 0.01 * len(xs)
    for x in [1.2231614256588297, 0.47938056872090196]:
        assert not is_correctly_rounded(x, lm(x))
        assert is_correctly_rounded(x, cr(x))


def _two_phase():
    cr = P.Oracle.load(cr_cos=True)
    f = cr.orc_cos_2phase
    f.restype = C.c_long
    f.argtypes = [C.c_void_p, C.c_long, C.c_void_p, C.c_void_p]

    def run(xs):
        xs = np.ascontiguousarray(xs, dtype=np.float64)
        out = np.empty_like(xs)
        slow = np.zeros(len(xs), dtype=np.uint8)
        ns = f(xs.ctypes.data, len(xs), out.ctypes.data, slow.ctypes.data)
        assert ns == int(slow.sum())
        return out, slow.astype(bool)
    return run


def _accurate(xs):
    cr, _ = _cos_fns()
    return np.array([cr(float(x)) for x in xs])


def test_two_phase_cosine_equals_the_accurate_one(oracle_built):
    """The CUDA path's two-phase cosine (quick double / double-double phase
    with a rounding test, accurate phase on failure) returns the same bits
    as the accurate double-double cosine: both are correctly rounded.  The
    quick phase decides all but a small fraction of arguments."""
    run = _two_phase()
    rng = np.random.default_rng(11)
    xs = np.concatenate([delta_args(200000, 12), rng.uniform(-4.0, 4.0, 100000),
                         rng.uniform(-1e-6, 1e-6, 2000),
                         (PI_T / 2) * np.array([0.0, 1.0, -1.0, 2.0, -2.0, 0.5, -0.5, 1.5, -1.5]),
                         np.array([math.pi / 2, -math.pi / 2, math.pi, -math.pi, math.pi / 4,
                                   3 * math.pi / 4, 1.2231614256588297, 0.47938056872090196,
                                   -2.1501599567293868, 1.7759313193883071])])
    # arguments next to k pi/4 (the reduction's switch points and the range ends)
    near = []
    for m in range(-5, 6):
        v = m * math.pi / 4
        for _ in range(20):
            near += [v, -v]
            v = math.nextafter(v, math.inf)
    xs = np.concatenate([xs, np.array(near)])
    out, slow = run(xs)
    ref = _accurate(xs)
    bad = np.nonzero(out.view(np.int64) != ref.view(np.int64))[0]
    assert bad.size == 0, [(xs[i], out[i], ref[i]) for i in bad[:5]]
    assert 0 < slow.sum() < 2e-3 * len(xs), slow.sum()


def test_two_phase_fallback_cases_are_correctly_rounded(oracle_built):
    """The arguments the rounding test leaves to the accurate phase are the
    ones whose cosine lies close to a rounding boundary; among 400k
    delta-kernel arguments each of them comes out correctly rounded by the
    60-digit evaluation, as do the quick phase's results on a sample."""
    run = _two_phase()
    xs = delta_args(400000, 21)
    out, slow = run(xs)
    idx = np.nonzero(slow)[0]
    assert 0 < idx.size < 400
    for i in list(idx) + list(range(200)):
        assert is_correctly_rounded(float(xs[i]), float(out[i])), xs[i]
