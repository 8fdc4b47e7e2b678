"""Double and complex level-2 routines through the C ABI against the oracle.

DGEMV / CGEMV / ZGEMV (dgemv.rs, cgemv.rs:60-80, zgemv.rs): every op (N, T,
and C for complex), ragged sizes around the 128-row strips, padded lda,
strided x / y, real and complex beta (the reference scales by csscal/zdscal
when Im(beta) == 0, by cscal/zscal otherwise), alpha == 0 (beta step only) and
the quick return.  The bound is component-wise, |y - y_oracle| <=
tol (|alpha| |op(A)||x| + |beta||y|), with tol 1e-5 for complex64 (the
fp32 tolerance of sgemv_tests.rs) and 1e-13 for double data.
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle

pytestmark = pytest.mark.gpu

SIZES = [(1, 1), (7, 5), (127, 130), (128, 64), (129, 257), (300, 1000), (2049, 33), (5000, 4100)]
TOL = {np.float64: 1e-13, np.complex64: 1e-5, np.complex128: 1e-13}


def rnd(rng, shape, dt):
    if np.issubdtype(dt, np.complexfloating):
        return (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(dt)
    return rng.uniform(-1, 1, shape).astype(dt)


def run_gemv(dt, trans, m, n, lda, incx, incy, alpha, beta, seed, nan_y=False):
    rng = np.random.default_rng(seed)
    a = rnd(rng, (n, lda), dt)                       # [col][row]
    xlen, ylen = (m, n) if trans else (n, m)
    x = rnd(rng, (xlen - 1) * incx + 1, dt)
    y = rnd(rng, (ylen - 1) * incy + 1, dt)
    if nan_y:
        y[::incy][0] = np.nan
    Y = torch.from_numpy(y.copy()).cuda()
    fn = {np.float64: cb.dgemv, np.complex64: cb.cgemv, np.complex128: cb.zgemv}[dt]
    fn(trans, m, n, alpha, torch.from_numpy(a.ravel()).cuda(), lda, torch.from_numpy(x).cuda(), incx,
       beta, Y, incy)
    torch.cuda.synchronize()
    got = Y.cpu().numpy()
    orc = {np.float64: oracle.dgemv, np.complex64: oracle.cgemv, np.complex128: oracle.zgemv}[dt]
    want = orc(trans, m, n, alpha, a.ravel(), lda, x, incx, beta, y, incy)
    # scale: |alpha| |op(A)| |x| + |beta| |y|
    A = np.abs(a[:, :m].T.astype(np.complex128))
    opA = A if trans == 0 else A.T
    scale = abs(alpha) * (opA @ np.abs(x[::incx][:xlen])) + abs(beta) * np.abs(y[::incy][:ylen])
    g = got[::incy][:ylen]
    fin = np.isfinite(want)
    np.testing.assert_array_equal(np.isnan(g), np.isnan(want))
    assert (np.abs(g[fin] - want[fin]) <= TOL[dt] * scale[fin] + 1e-30).all(), np.abs(g - want).max()
    # stride holes untouched
    if incy > 1:
        holes = np.arange(y.size) % incy != 0
        np.testing.assert_array_equal(got[holes], y[holes])


@pytest.mark.parametrize("m,n", SIZES)
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_dgemv(cuda, m, n, trans):
    run_gemv(np.float64, trans, m, n, m + 3, 1, 1, 1.5, 0.5, m * 7 + n + trans)


@pytest.mark.parametrize("m,n", SIZES)
@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("dt", [np.complex64, np.complex128], ids=["c", "z"])
def test_cz_gemv(cuda, dt, m, n, trans):
    run_gemv(dt, trans, m, n, m + 2, 1, 1, 1.5 - 0.25j, 0.5 + 0.75j, m * 7 + n + trans)


@pytest.mark.parametrize("dt", [np.float64, np.complex64, np.complex128], ids=["d", "c", "z"])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_gemv_strides_and_beta_modes(cuda, dt, trans):
    cplx = np.issubdtype(dt, np.complexfloating)
    run_gemv(dt, trans, 300, 211, 305, 3, 2, 0.75 + (0.5j if cplx else 0), 1.0, 11 + trans)   # beta == 1
    run_gemv(dt, trans, 300, 211, 300, 1, 3, 2.0, -0.5, 12 + trans)                           # real beta
    # beta == 0 multiplies (scal): a NaN in y stays NaN, as in the reference
    run_gemv(dt, trans, 257, 129, 257, 2, 1, 1.25, 0.0, 13 + trans, nan_y=True)


@pytest.mark.parametrize("dt", [np.float64, np.complex64, np.complex128], ids=["d", "c", "z"])
def test_gemv_alpha_zero_and_quick_return(cuda, dt):
    run_gemv(dt, 0, 200, 100, 200, 1, 1, 0.0, 0.5, 21)      # beta step only
    run_gemv(dt, 1, 200, 100, 200, 1, 1, 0.0, 1.0, 22)      # no-op
