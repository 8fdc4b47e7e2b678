"""Fused level-1.5 updates through the C ABI against the oracle
(coral-aarch64/src/level1_special): saxpyf / daxpyf / caxpyf / zaxpyf
(y += A x), sdotf / ddotf / cdotuf / zdotuf (out += A^T x) and cdotcf / zdotcf
(out += A^H x).

The oracle is the GEMV restatement with alpha = beta = 1.  The bound is
component-wise, |y - y_oracle| <= tol (|op(A)||x| + |y|), with tol 1e-5 for
fp32 data (sgemv_tests.rs) and 1e-13 for fp64; stride holes of y stay
untouched; an empty matrix is a no-op whatever the pointers are.
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle

pytestmark = pytest.mark.gpu

DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
TOL = {"s": 1e-5, "d": 1e-13, "c": 1e-5, "z": 1e-13}
AXPYF = {"s": cb.saxpyf, "d": cb.daxpyf, "c": cb.caxpyf, "z": cb.zaxpyf}
DOTF = {("s", 1): cb.sdotf, ("d", 1): cb.ddotf, ("c", 1): cb.cdotuf, ("c", 2): cb.cdotcf,
        ("z", 1): cb.zdotuf, ("z", 2): cb.zdotcf}
SIZES = [(1, 1), (7, 5), (128, 8), (129, 257), (300, 1000), (2049, 33), (4096, 4096)]


def rnd(rng, shape, kind):
    dt = DT[kind]
    if kind in "sd":
        return rng.uniform(-1, 1, shape).astype(dt)
    return (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(dt)


def want_gemv(kind, op, m, n, a, lda, x, incx, y, incy):
    if kind == "s":
        return oracle.sgemv(min(op, 1), m, n, 1.0, a, lda, x, incx, 1.0, y, incy)
    if kind == "d":
        return oracle.dgemv(min(op, 1), m, n, 1.0, a, lda, x, incx, 1.0, y, incy)
    fn = oracle.cgemv if kind == "c" else oracle.zgemv
    return fn(op, m, n, 1.0, a, lda, x, incx, 1.0, y, incy)


def run(kind, op, m, n, lda, incx, incy, seed):
    rng = np.random.default_rng(seed)
    a = rnd(rng, (n, lda), kind)
    xlen, ylen = (n, m) if op == 0 else (m, n)
    x = rnd(rng, (xlen - 1) * incx + 1, kind)
    y = rnd(rng, (ylen - 1) * incy + 1, kind)
    Y = torch.from_numpy(y.copy()).cuda()
    A = torch.from_numpy(a.ravel()).cuda()
    X = torch.from_numpy(x).cuda()
    if op == 0:
        AXPYF[kind](m, n, X, incx, A, lda, Y, incy)
    else:
        DOTF[(kind, op)](m, n, A, lda, X, incx, Y)
    torch.cuda.synchronize()
    got = Y.cpu().numpy()
    want = want_gemv(kind, op, m, n, a.ravel(), lda, x, incx, y, incy)
    absA = np.abs(a[:, :m].T.astype(np.complex128))
    opA = absA if op == 0 else absA.T
    scale = opA @ np.abs(x[::incx][:xlen]) + np.abs(y[::incy][:ylen])
    g = got[::incy][:ylen]
    assert (np.abs(g - want) <= TOL[kind] * scale + 1e-30).all(), np.abs(g - want).max()
    if incy > 1:
        holes = np.arange(y.size) % incy != 0
        np.testing.assert_array_equal(got[holes], y[holes])


@pytest.mark.parametrize("kind", "sdcz")
@pytest.mark.parametrize("m,n", SIZES)
def test_axpyf(cuda, kind, m, n):
    run(kind, 0, m, n, m + 3, 1, 1, m + 3 * n)


@pytest.mark.parametrize("kind,op", list(DOTF))
@pytest.mark.parametrize("m,n", SIZES)
def test_dotf(cuda, kind, op, m, n):
    run(kind, op, m, n, m + 1, 1, 1, m + 5 * n + op)


@pytest.mark.parametrize("kind", "sdcz")
def test_strided(cuda, kind):
    run(kind, 0, 300, 211, 305, 3, 2, 1)          # strided x and y (saxpy-per-column path of the reference)
    run(kind, 1, 300, 211, 300, 2, 1, 2)          # strided x (scalar strided dots)
    if kind in "cz":
        run(kind, 2, 257, 129, 260, 3, 1, 3)


def test_quick_return_and_bad_args(cuda):
    cb.saxpyf(0, 5, None, 1, None, 1, None, 1)
    cb.zdotcf(5, 0, None, 1, None, 1, None)
    a = torch.zeros(16, dtype=torch.float64, device="cuda")
    with pytest.raises(cb.CoralError) as e:
        cb.daxpyf(4, 4, a, 0, a, 4, a, 1)
    assert e.value.bad_arg == 4
    with pytest.raises(cb.CoralError) as e:
        cb.ddotf(4, 4, a, 3, a, 1, a)
    assert e.value.bad_arg == 4
