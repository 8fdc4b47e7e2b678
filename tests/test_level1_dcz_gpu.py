"""Double and complex level 1 through the C ABI against the oracle
(coral-aarch64/src/level1: d/c/z dot, asum, nrm2, i?amax, axpy, scal incl.
csscal / zdscal, copy, swap, the rotations and the rotation constructors).

Bit-exact: i?amax (index), axpy, scal, copy, swap, rot, rotm, rotg, rotmg --
the oracle reproduces the reference's NEON-body / scalar-tail roundings.
Tolerance: dot, asum, nrm2 within the reference tests' own bounds
(dot_tests.rs:176-179, asum_tests.rs:106-109, nrm2_tests.rs:106-109);
the GPU sums in fp64 (fp32 data) or fp64 (fp64 data), the oracle in
double-double / long double.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import coral_b200 as cb
import fixtures as fx
import oracle
from coral_b200.blas import handle

pytestmark = pytest.mark.gpu
DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
SIZES = [1, 2, 3, 5, 8, 13, 1000, 4096 + 3, (1 << 20) + 5]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def rnd(kind, n, seed, lo=-1.0, hi=1.0):
    rng = np.random.default_rng(seed)
    if kind in "sd":
        return rng.uniform(lo, hi, n).astype(DT[kind])
    return (rng.uniform(lo, hi, n) + 1j * rng.uniform(lo, hi, n)).astype(DT[kind])


def tol(kind, fn=""):
    if kind in "sc":
        return (4e-6, 4e-6) if fn.startswith("dot") else (1e-6, 1e-6)
    return 1e-12, 1e-12


def close(got, want, kind, fn=""):
    rtol, atol = tol(kind, fn)
    got, want = complex(got), complex(want)
    assert abs(got - want) <= atol + rtol * max(abs(got), abs(want)), (got, want)


DOT = {("d", 0): cb.ddot, ("c", 0): cb.cdotu, ("c", 1): cb.cdotc, ("z", 0): cb.zdotu, ("z", 1): cb.zdotc}
ASUM = {"s": cb.sasum, "d": cb.dasum, "c": cb.scasum, "z": cb.dzasum}
NRM2 = {"d": cb.dnrm2, "c": cb.scnrm2, "z": cb.dznrm2}
IAMAX = {"d": cb.idamax, "c": cb.icamax, "z": cb.izamax}
AXPY = {"d": cb.daxpy, "c": cb.caxpy, "z": cb.zaxpy}
SCAL = {"d": cb.dscal, "c": cb.cscal, "z": cb.zscal}
RSCAL = {"c": cb.csscal, "z": cb.zdscal}
COPY = {"d": cb.dcopy, "c": cb.ccopy, "z": cb.zcopy}
SWAP = {"d": cb.dswap, "c": cb.cswap, "z": cb.zswap}
ROT = {"s": cb.srot, "d": cb.drot, "c": cb.csrot, "z": cb.zdrot}
ROTM = {"s": cb.srotm, "d": cb.drotm}


# ---- the reference's fixture cases ----------------------------------------------
@pytest.mark.parametrize("ci", range(len(fx.L1_CASES)))
def test_fixture_cases(cuda, ci):
    case = fx.L1_CASES[ci]
    kind, n, fn = case["kind"], case["n"], case["fn"]
    x, y = fx.l1_vectors(case)
    incx, incy = case["incx"], case.get("incy", 1)
    X = dev(x)
    Y = dev(y) if y is not None else None
    if fn == "axpy":
        AXPY[kind](n, case["alpha"], X, incx, Y, incy)
        np.testing.assert_array_equal(host(Y), oracle.axpy(kind, n, case["alpha"], x, incx, y, incy))
    elif fn == "scal":
        SCAL[kind](n, case["alpha"], X, incx)
        np.testing.assert_array_equal(host(X), oracle.scal(kind, n, case["alpha"], x, incx))
    elif fn == "sscal_r":
        RSCAL[kind](n, case["alpha"], X, incx)
        np.testing.assert_array_equal(host(X), oracle.scal(kind, n, case["alpha"], x, incx, real_alpha=True))
    elif fn in ("dotu", "dotc"):
        conj = int(fn == "dotc")
        close(DOT[(kind, conj)](n, X, incx, Y, incy), oracle.dot(kind, conj, n, x, incx, y, incy), kind, fn)
    elif fn == "asum":
        close(ASUM[kind](n, X, incx), oracle.asum(kind, n, x, incx), kind)
    elif fn == "nrm2":
        close(NRM2[kind](n, X, incx), oracle.nrm2(kind, n, x, incx), kind)
    elif fn == "iamax":
        assert IAMAX[kind](n, X, incx) == oracle.iamax(kind, n, x, incx)
    elif fn == "rot":
        c, s = fx.rot_cs(case)
        ROT[kind](n, X, incx, Y, incy, c, s)
        wx, wy = oracle.rot(kind, n, x, incx, y, incy, c, s)
        np.testing.assert_array_equal(host(X), wx)
        np.testing.assert_array_equal(host(Y), wy)
    elif fn == "rotm":
        ROTM[kind](n, X, incx, Y, incy, case["param"])
        wx, wy = oracle.rotm(kind, n, x, incx, y, incy, case["param"])
        np.testing.assert_array_equal(host(X), wx)
        np.testing.assert_array_equal(host(Y), wy)


# ---- reductions -------------------------------------------------------------------
@pytest.mark.parametrize("kind,conj", list(DOT))
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [(1, 1), (3, 2)])
def test_dot(cuda, kind, conj, n, inc):
    incx, incy = inc
    x = rnd(kind, (n - 1) * incx + 1, n)
    y = rnd(kind, (n - 1) * incy + 1, n + 1)
    got = DOT[(kind, conj)](n, dev(x), incx, dev(y), incy)
    want = oracle.dot(kind, conj, n, x, incx, y, incy)
    # relative to sum |x||y| (cancellation-safe bound of the summation error)
    scale = float(np.sum(np.abs(x[::incx][:n]).astype(np.float64) * np.abs(y[::incy][:n])))
    bound = 1e-6 * scale if kind == "c" else 1e-13 * scale
    assert abs(complex(got) - want) <= bound + 1e-300, (got, want, bound)


@pytest.mark.parametrize("kind", "sdcz")
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [1, 3])
def test_asum(cuda, kind, n, inc):
    x = rnd(kind, (n - 1) * inc + 1, 7 * n + inc)
    close(ASUM[kind](n, dev(x), inc), oracle.asum(kind, n, x, inc), kind)


@pytest.mark.parametrize("kind", "dcz")
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [1, 4])
def test_nrm2(cuda, kind, n, inc):
    x = rnd(kind, (n - 1) * inc + 1, 11 * n + inc)
    close(NRM2[kind](n, dev(x), inc), oracle.nrm2(kind, n, x, inc), kind)


@pytest.mark.parametrize("kind", "dz")
@pytest.mark.parametrize("mag", [1e200, 1e-200, 1e-300, 1e300])
def test_nrm2_rescaled(cuda, kind, mag):
    """Sums of squares that overflow / underflow fp64 take the rescaled pass."""
    n = 10007
    x = (rnd(kind, n, 5) * mag).astype(DT[kind])
    got = NRM2[kind](n, dev(x), 1)
    want = oracle.nrm2(kind, n, x, 1)
    assert np.isfinite(got) and got > 0
    assert abs(got - want) <= 1e-12 * want


@pytest.mark.parametrize("kind", "dcz")
def test_nrm2_nan_inf_and_quick_returns(cuda, kind):
    x = rnd(kind, 4099, 3)
    y = x.copy()
    y[1234] = np.inf
    assert NRM2[kind](4099, dev(y), 1) == np.inf
    y[77] = np.nan
    assert np.isnan(NRM2[kind](4099, dev(y), 1))   # NaN wins over inf
    assert NRM2[kind](0, dev(x), 1) == 0.0
    assert NRM2[kind](5, dev(x), 0) == 0.0
    assert ASUM[kind](5, dev(x), 0) == 0.0


@pytest.mark.parametrize("kind", "dcz")
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [1, 3])
def test_iamax(cuda, kind, n, inc):
    x = rnd(kind, (n - 1) * inc + 1, 13 * n + inc)
    if n > 4:   # a planted tie: the first occurrence wins
        v = x[::inc][n // 3] * 0 + (50 if kind == "d" else 30 + 20j)
        x[(n // 3) * inc] = v
        x[(2 * n // 3) * inc] = np.conj(v) if kind != "d" else -v
    assert IAMAX[kind](n, dev(x), inc) == oracle.iamax(kind, n, x, inc)


@pytest.mark.parametrize("kind", "dcz")
def test_iamax_nan(cuda, kind):
    x = rnd(kind, 3000, 9)
    x[5] = np.nan
    x[2999] = 100
    assert IAMAX[kind](3000, dev(x), 1) == 2999 == oracle.iamax(kind, 3000, x, 1)
    allnan = np.full(777, np.nan, DT[kind])
    assert IAMAX[kind](777, dev(allnan), 1) == 0
    assert IAMAX[kind](0, dev(x), 1) == 0 and IAMAX[kind](5, dev(x), 0) == 0


# ---- elementwise -----------------------------------------------------------------
@pytest.mark.parametrize("kind", "dcz")
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [(1, 1), (2, 3)])
def test_axpy_bit_exact(cuda, kind, n, inc):
    incx, incy = inc
    x = rnd(kind, (n - 1) * incx + 1, n)
    y = rnd(kind, (n - 1) * incy + 1, n + 2)
    alpha = 0.37 if kind == "d" else 0.37 - 1.21j
    Y = dev(y)
    AXPY[kind](n, alpha, dev(x), incx, Y, incy)
    np.testing.assert_array_equal(host(Y), oracle.axpy(kind, n, alpha, x, incx, y, incy))


@pytest.mark.parametrize("kind", "dcz")
def test_axpy_zero_alpha_untouched(cuda, kind):
    x = np.full(100, np.nan, DT[kind])
    y = rnd(kind, 100, 1)
    Y = dev(y)
    AXPY[kind](100, 0.0, dev(x), 1, Y, 1)
    np.testing.assert_array_equal(host(Y), y)


@pytest.mark.parametrize("kind", "dcz")
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [1, 3])
def test_scal_bit_exact(cuda, kind, n, inc):
    x = rnd(kind, (n - 1) * inc + 1, n + 5)
    alpha = -1.7 if kind == "d" else 0.6 + 0.8j
    X = dev(x)
    SCAL[kind](n, alpha, X, inc)
    np.testing.assert_array_equal(host(X), oracle.scal(kind, n, alpha, x, inc))
    if kind != "d":
        X = dev(x)
        RSCAL[kind](n, -1.7, X, inc)
        np.testing.assert_array_equal(host(X), oracle.scal(kind, n, -1.7, x, inc, real_alpha=True))


@pytest.mark.parametrize("kind", "dcz")
def test_scal_zero_multiplies(cuda, kind):
    x = rnd(kind, 64, 2)
    x[3] = np.nan
    X = dev(x)
    SCAL[kind](64, 0.0, X, 1)
    got = host(X)
    assert np.isnan(got[3]) and (got[np.arange(64) != 3] == 0).all()


@pytest.mark.parametrize("kind", "dcz")
@pytest.mark.parametrize("n", [1, 7, 4096 + 3, (1 << 20) + 5])
@pytest.mark.parametrize("inc", [(1, 1), (3, 2)])
def test_copy_swap(cuda, kind, n, inc):
    incx, incy = inc
    x = rnd(kind, (n - 1) * incx + 1, n)
    y = rnd(kind, (n - 1) * incy + 1, n + 1)
    Y = dev(y)
    COPY[kind](n, dev(x), incx, Y, incy)
    np.testing.assert_array_equal(host(Y), oracle.copy(n, x, incx, y, incy))
    X, Y = dev(x), dev(y)
    SWAP[kind](n, X, incx, Y, incy)
    wx, wy = oracle.swap(n, x, incx, y, incy)
    np.testing.assert_array_equal(host(X), wx)
    np.testing.assert_array_equal(host(Y), wy)


@pytest.mark.parametrize("kind", "sdcz")
@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [(1, 1), (2, 3)])
def test_rot_bit_exact(cuda, kind, n, inc):
    incx, incy = inc
    x = rnd(kind, (n - 1) * incx + 1, n)
    y = rnd(kind, (n - 1) * incy + 1, n + 3)
    real = np.float32 if kind in "sc" else np.float64
    c, s = real(np.cos(real(0.7))), real(np.sin(real(0.7)))
    X, Y = dev(x), dev(y)
    ROT[kind](n, X, incx, Y, incy, c, s)
    wx, wy = oracle.rot(kind, n, x, incx, y, incy, c, s)
    np.testing.assert_array_equal(host(X), wx)
    np.testing.assert_array_equal(host(Y), wy)


@pytest.mark.parametrize("kind", "sd")
@pytest.mark.parametrize("flag", [-1.0, 0.0, 1.0, 0.5, -2.0])
@pytest.mark.parametrize("n,inc", [(1, (1, 1)), (7, (1, 1)), (1027, (1, 1)), (4099, (2, 3)), ((1 << 20) + 3, (1, 1))])
def test_rotm_bit_exact(cuda, kind, flag, n, inc):
    incx, incy = inc
    x = rnd(kind, (n - 1) * incx + 1, n)
    y = rnd(kind, (n - 1) * incy + 1, n + 1)
    param = [flag, 1.1, -0.45, 0.7, 0.93]
    X, Y = dev(x), dev(y)
    ROTM[kind](n, X, incx, Y, incy, param)
    wx, wy = oracle.rotm(kind, n, x, incx, y, incy, param)
    np.testing.assert_array_equal(host(X), wx)
    np.testing.assert_array_equal(host(Y), wy)


# ---- rotation constructors ---------------------------------------------------------
ROTG_EXTRA = [(1.0, 1.0), (-1e-30, 3e-30), (6.0, -6.0), (0.0, 0.0), (1e20, -3e19), (-0.0, 2.5)]


@pytest.mark.parametrize("kind", "sd")
@pytest.mark.parametrize("ab", fx.ROTG_CASES + ROTG_EXTRA)
def test_rotg_bit_exact(cuda, kind, ab):
    fn = cb.srotg if kind == "s" else cb.drotg
    real = np.float32 if kind == "s" else np.float64
    a, b = real(ab[0]), real(ab[1])
    assert fn(a, b) == tuple(real(v) for v in oracle.rotg(kind, a, b))


ROTMG_EXTRA = [(1.0, 1.0, 1.0, 1.0), (2.0, 0.0, 1.0, 3.0), (-1.0, 2.0, 3.0, 4.0), (1e-9, 1e9, 3.0, 2.0),
               (1e8, 1e-8, 1e-3, 5.0), (3.0, -2.0, 1.0, 5.0), (4.0, 2.0, 1e-4, 1e4)]


@pytest.mark.parametrize("case", fx.ROTMG_CASES + [(k,) + e for k in "sd" for e in ROTMG_EXTRA])
def test_rotmg_bit_exact(cuda, case):
    kind, d1, d2, x1, y1 = case
    real = np.float32 if kind == "s" else np.float64
    fn = cb.srotmg if kind == "s" else cb.drotmg
    g = fn(real(d1), real(d2), real(x1), real(y1))
    w = oracle.rotmg(kind, real(d1), real(d2), real(x1), real(y1))
    if w[3][0] == -2.0:   # d2 y1 == 0: only the flag is written
        assert g[3][0] == -2.0 and g[:3] == tuple(real(v) for v in (d1, d2, x1))
        return
    assert g[:3] == tuple(real(v) for v in w[:3])
    assert [real(v) for v in g[3]] == [real(v) for v in w[3]]


# ---- device pointer mode -----------------------------------------------------------
def test_device_pointer_mode(cuda):
    h = handle()
    x = rnd("z", 5000, 1)
    y = rnd("z", 5000, 2)
    X, Y = dev(x), dev(y)
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    idx = torch.zeros(1, dtype=torch.int64, device="cuda")
    rot = torch.tensor([3.0, 4.0, 0.0, 0.0], dtype=torch.float64, device="cuda")
    p = lambda t, off=0: C.c_void_p(t.data_ptr() + 8 * off)  # noqa: E731
    h.set_pointer_mode(1)
    try:
        h.call("coral_zdotc", 5000, p(X), 1, p(Y), 1, p(out, 0))
        h.call("coral_dznrm2", 5000, p(X), 1, p(out, 2))
        h.call("coral_izamax", 5000, p(X), 1, p(idx))
        h.call("coral_drotg", p(rot, 0), p(rot, 1), p(rot, 2), p(rot, 3))
    finally:
        h.set_pointer_mode(0)
    o = host(out)
    close(complex(o[0], o[1]), oracle.dot("z", 1, 5000, x, 1, y, 1), "z")
    close(o[2], oracle.nrm2("z", 5000, x, 1), "z")
    assert int(host(idx)[0]) == oracle.iamax("z", 5000, x, 1)
    assert tuple(host(rot)) == oracle.rotg("d", 3.0, 4.0)


# ---- argument checks -----------------------------------------------------------------
def test_bad_arguments(cuda):
    x = dev(rnd("z", 16, 1))
    with pytest.raises(cb.CoralError) as e:
        cb.zdotc(4, x, 0, x, 1)
    assert e.value.bad_arg == 3
    with pytest.raises(cb.CoralError) as e:
        cb.zaxpy(4, 1.0, x, 1, x, 0)
    assert e.value.bad_arg == 6
    with pytest.raises(cb.CoralError) as e:   # complex128 data must be 16-byte aligned
        handle().call("coral_zdrot", 2, C.c_void_p(x.data_ptr() + 8), 1, C.c_void_p(x.data_ptr()), 1,
                      C.c_double(0.5), C.c_double(0.5))
    assert e.value.bad_arg == 2
    # quick returns before any pointer check
    cb.zaxpy(0, 1.0, None, 1, None, 1)
    cb.zscal(5, 2.0, None, 0)
    cb.drotm(0, None, 1, None, 1, [-1, 1, 2, 3, 4])
    assert cb.zdotu(0, None, 1, None, 1) == 0
