"""Host-slice drop-ins for the rest of the hot path: ssymv, chemv, strmv,
sger, ssyr, ssyr2, snrm2, scopy, sswap, sscal, dgemm, cgemm, zgemm.

Each takes the reference's own argument list over host memory
(ssymv.rs:99-110, chemv.rs:96-107, strmv.rs:59-73, sger.rs:68-78,
ssyr.rs:63-71, ssyr2.rs:59-69, snrm2.rs:45, scopy.rs:28, sswap.rs:35,
sscal.rs:30, dgemm.rs:107, cgemm.rs:127-157, zgemm.rs:123), copies in,
computes on the GPU and copies back.  Each result is compared with the device
entry point on the same inputs (bit for bit: the same kernels run) and, for
the bit-exact routines, with the oracle; stride holes and leading-dimension
padding must come back unchanged, and a bad argument is rejected before any
copy.
"""
import ctypes

import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle
from coral_b200 import _lib

pytestmark = pytest.mark.gpu
vp = ctypes.c_void_p


def P(a):
    return vp(a.ctypes.data)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def rnd(n, seed, dtype=np.float32):
    rng = np.random.default_rng(seed)
    if np.issubdtype(dtype, np.complexfloating):
        return (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(dtype)
    return rng.uniform(-1, 1, n).astype(dtype)


def cpair(z, dt):
    return (dt * 2)(z.real, z.imag)


@pytest.mark.parametrize("uplo", [0, 1])
def test_host_ssymv_chemv(cuda, uplo):
    lib = _lib.load()
    n, lda, inc = 777, 781, 2
    a = rnd(lda * n, 1)
    x = rnd((n - 1) * inc + 1, 2)
    y = rnd((n - 1) * inc + 1, 3)
    yh = y.copy()
    assert lib.coral_host_ssymv(uplo, n, 1.5, P(a), lda, P(x), inc, 0.5, P(yh), inc) == 0
    Y = dev(y)
    cb.ssymv(uplo, n, 1.5, dev(a), lda, dev(x), inc, 0.5, Y, inc)
    np.testing.assert_array_equal(yh, host(Y))
    ac = rnd(lda * n, 4, np.complex64)
    xc = rnd((n - 1) * inc + 1, 5, np.complex64)
    yc = rnd((n - 1) * inc + 1, 6, np.complex64)
    ych = yc.copy()
    al, be = 1.5 - 0.5j, 0.25 + 1j
    assert lib.coral_host_chemv(uplo, n, cpair(al, ctypes.c_float), P(ac), lda, P(xc), inc,
                                cpair(be, ctypes.c_float), P(ych), inc) == 0
    Yc = dev(yc)
    cb.chemv(uplo, n, al, dev(ac), lda, dev(xc), inc, be, Yc, inc)
    np.testing.assert_array_equal(ych, host(Yc))


@pytest.mark.parametrize("trans", [0, 1])
def test_host_strmv(cuda, trans):
    lib = _lib.load()
    n, lda, inc = 500, 503, 3
    a = rnd(lda * n, 7)
    x = rnd((n - 1) * inc + 1, 8)
    xh = x.copy()
    assert lib.coral_host_strmv(1, trans, 1, n, P(a), lda, P(xh), inc) == 0
    X = dev(x)
    cb.strmv(1, trans, 1, n, dev(a), lda, X, inc)
    np.testing.assert_array_equal(xh, host(X))
    holes = np.arange(x.size) % inc != 0
    np.testing.assert_array_equal(xh[holes], x[holes])


def test_host_rank_updates_bit_exact(cuda):
    lib = _lib.load()
    m, n, lda = 300, 257, 305
    x, y = rnd(m, 9), rnd(n, 10)
    a = rnd(lda * n, 11)
    ah = a.copy()
    assert lib.coral_host_sger(m, n, 0.75, P(x), 1, P(y), 1, P(ah), lda) == 0
    np.testing.assert_array_equal(ah, oracle.sger(m, n, 0.75, x, 1, y, 1, a, lda))
    sq = rnd(lda * n, 12)
    xs = rnd(n, 13)
    for uplo in (0, 1):
        sh = sq.copy()
        assert lib.coral_host_ssyr(uplo, n, -1.25, P(xs), 1, P(sh), lda) == 0
        np.testing.assert_array_equal(sh, oracle.ssyr(uplo, n, -1.25, xs, 1, sq, lda))
        sh2 = sq.copy()
        assert lib.coral_host_ssyr2(uplo, n, 0.5, P(xs), 1, P(y), 1, P(sh2), lda) == 0
        np.testing.assert_array_equal(sh2, oracle.ssyr2(uplo, n, 0.5, xs, 1, y, 1, sq, lda))


def test_host_level1(cuda):
    lib = _lib.load()
    n, inc = 100003, 2
    x = rnd((n - 1) * inc + 1, 14)
    y = rnd((n - 1) * inc + 1, 15)
    r = ctypes.c_float()
    assert lib.coral_host_snrm2(n, P(x), inc, ctypes.byref(r)) == 0
    assert r.value == cb.snrm2(n, dev(x), inc)
    assert abs(r.value - oracle.snrm2(n, x, inc)) <= 1e-6 * oracle.snrm2(n, x, inc)
    yc = y.copy()
    assert lib.coral_host_scopy(n, P(x), inc, P(yc), inc) == 0
    np.testing.assert_array_equal(yc, oracle.scopy(n, x, inc, y, inc))
    xs, ys = x.copy(), y.copy()
    assert lib.coral_host_sswap(n, P(xs), inc, P(ys), inc) == 0
    wx, wy = oracle.sswap(n, x, inc, y, inc)
    np.testing.assert_array_equal(xs, wx)
    np.testing.assert_array_equal(ys, wy)
    xc = x.copy()
    assert lib.coral_host_sscal(n, 0.3, P(xc), inc) == 0
    np.testing.assert_array_equal(xc, oracle.sscal(n, 0.3, x, inc))


@pytest.mark.parametrize("mode", [0, 2], ids=["native", "ozaki_int8"])
def test_host_dgemm(cuda, mode):
    lib = _lib.load()
    m, n, k, lda, ldb, ldc = 300, 200, 150, 150, 151, 305   # op_a = T, op_b = N
    a, b, c = rnd(lda * m, 16, np.float64), rnd(ldb * n, 17, np.float64), rnd(ldc * n, 18, np.float64)
    ch = c.copy()
    assert lib.coral_host_set_gemm_mode(mode) == 0
    try:
        assert lib.coral_host_dgemm(1, 0, m, n, k, 1.5, P(a), lda, P(b), ldb, 0.0, P(ch), ldc) == 0
    finally:
        lib.coral_host_set_gemm_mode(0)
    ii, jj = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
    want, bound = oracle.gemm_sample(1, 0, m, n, k, 1.5, a, lda, b, ldb, 0.0, c, ldc, ii.ravel(), jj.ravel())
    got = ch.reshape(n, ldc).T
    assert (np.abs(got[:m].ravel() - want) <= 1e-13 * bound).all()
    np.testing.assert_array_equal(got[m:], c.reshape(n, ldc).T[m:])  # padding untouched, beta == 0


@pytest.mark.parametrize("cplx", [np.complex64, np.complex128])
def test_host_cgemm_zgemm(cuda, cplx):
    lib = _lib.load()
    m, n, k, lda, ldb, ldc = 130, 70, 90, 133, 72, 131   # op_a = N, op_b = C
    a, b, c = rnd(lda * k, 19, cplx), rnd(ldb * k, 20, cplx), rnd(ldc * n, 21, cplx)
    ch = c.copy()
    fn = lib.coral_host_cgemm if cplx == np.complex64 else lib.coral_host_zgemm
    dt = ctypes.c_float if cplx == np.complex64 else ctypes.c_double
    al, be = 0.5 + 1j, -0.25 + 0.5j
    assert fn(0, 2, m, n, k, cpair(al, dt), P(a), lda, P(b), ldb, cpair(be, dt), P(ch), ldc) == 0
    ii, jj = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
    want, bound = oracle.gemm_sample(0, 2, m, n, k, al, a, lda, b, ldb, be, c, ldc, ii.ravel(), jj.ravel())
    got = ch.reshape(n, ldc).T
    tol = 1e-5 if cplx == np.complex64 else 1e-13
    assert (np.abs(got[:m].ravel() - want) <= tol * bound).all()
    np.testing.assert_array_equal(got[m:], c.reshape(n, ldc).T[m:])


def test_host_slices_reject_bad_args_before_copies(cuda):
    lib = _lib.load()
    a = np.zeros(64, np.float32)
    assert lib.coral_host_ssymv(0, 8, 1.0, P(a), 4, P(a), 1, 0.0, P(a), 1) == 1   # lda < n
    assert lib.coral_host_strmv(0, 3, 1, 4, P(a), 4, P(a), 1) == 1                # bad trans
    assert lib.coral_host_sger(4, 4, 1.0, P(a), 0, P(a), 1, P(a), 4) == 1          # incx == 0
    assert lib.coral_host_ssyr2(2, 4, 1.0, P(a), 1, P(a), 1, P(a), 4) == 1         # bad uplo
    assert lib.coral_host_dgemm(0, 0, 4, 4, 4, 1.0, P(a), 2, P(a), 4, 0.0, P(a), 4) == 1
    assert lib.coral_host_scopy(0, None, 1, None, 1) == 0                          # n == 0
