"""Level-2 parity through the C ABI (coral-aarch64/src/level2).

SGEMV against the oracle (fp64) with the reference's tolerance 1e-5
(tests/level2/sgemv_tests.rs:116-117) and against the golden CBLAS outputs of
the reference's own fixture cases; SGER/SSYR/SSYR2 bit-exact.
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import fixtures as fx
import oracle
from conftest import allclose_ref

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def rnd(n, seed):
    return np.random.default_rng(seed).uniform(-1, 1, n).astype(np.float32)


def test_sgemv_reference_fixtures(cuda, golden):
    for si, (m, n, lda, strides) in enumerate(fx.GEMV_SHAPES):
        a = fx.gemv_matrix(m, n, lda)
        A = dev(a)
        for (incx, incy) in strides:
            for trans in (0, 1):
                xl, yl = (n, m) if trans == 0 else (m, n)
                x = fx.gemv_x(xl, incx)
                y0 = fx.gemv_y(yl, incy)
                for ci, (alpha, beta) in enumerate(fx.GEMV_COEFFS):
                    Y = dev(y0)
                    cb.sgemv(trans, m, n, alpha, A, lda, dev(x), incx, beta, Y, incy)
                    got = host(Y)[::incy][:yl]
                    allclose_ref(got, golden[f"sgemv_s{si}_{incx}{incy}_t{trans}_c{ci}"], 1e-5, 1e-5)
                    assert np.array_equal(host(Y)[np.arange(len(y0)) % incy != 0],
                                          y0[np.arange(len(y0)) % incy != 0])


GEMV_CASES = [
    (1, 1, 1), (5, 4, 5), (33, 17, 40), (128, 128, 128), (129, 300, 131), (1000, 7, 1003),
    (7, 1000, 7), (4097, 513, 4100), (8192, 8192, 8192), (20000, 64, 20000), (64, 20000, 64),
]


@pytest.mark.parametrize("m,n,lda", GEMV_CASES)
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_sgemv_random(cuda, m, n, lda, trans):
    a = rnd(lda * n, m * 7 + n)
    t = trans != 0
    xl, yl = (m, n) if t else (n, m)
    x, y = rnd(xl, 1), rnd(yl, 2)
    for alpha, beta in [(1.5, 0.5), (1.0, 0.0), (-0.7, 1.0)]:
        Y = dev(y)
        cb.sgemv(trans, m, n, alpha, dev(a), lda, dev(x), 1, beta, Y, 1)
        want = oracle.sgemv(trans, m, n, alpha, a, lda, x, 1, beta, y, 1)
        # relative to the row/column scale: |error| <= 1e-5 * (|alpha| |A||x| + |beta y|)
        absA = np.abs(a.reshape(n, lda).T[:m, :].astype(np.float64))
        scale = np.abs(alpha) * ((absA.T if t else absA) @ np.abs(x)) + np.abs(beta * y)
        err = np.abs(host(Y) - want)
        assert (err <= 1e-5 * scale + 1e-6).all(), float((err / (scale + 1e-30)).max())


def test_sgemv_quick_returns_and_beta_semantics(cuda):
    a, x = rnd(16, 1), rnd(4, 2)
    y = np.array([1.0, np.nan, 2.0, 3.0], np.float32)
    Y = dev(y)
    cb.sgemv(0, 4, 4, 0.0, dev(a), 4, dev(x), 1, 1.0, Y, 1)  # alpha == 0 && beta == 1
    np.testing.assert_array_equal(host(Y), y)
    cb.sgemv(0, 4, 0, 2.0, dev(a), 4, dev(x), 1, 0.0, Y, 1)  # empty matrix
    np.testing.assert_array_equal(host(Y), y)
    cb.sgemv(0, 4, 4, 0.0, dev(a), 4, dev(x), 1, 0.0, Y, 1)  # beta == 0 multiplies (sscal)
    got = host(Y)
    assert np.isnan(got[1]) and got[0] == 0.0


def test_sgemv_bad_args(cuda):
    A = dev(rnd(16, 1))
    with pytest.raises(cb.CoralError) as e:
        cb.sgemv(0, 4, 4, 1.0, A, 3, A, 1, 0.0, A, 1)
    assert e.value.bad_arg == 6
    with pytest.raises(cb.CoralError) as e:
        cb.sgemv(7, 4, 4, 1.0, A, 4, A, 1, 0.0, A, 1)
    assert e.value.bad_arg == 1


@pytest.mark.parametrize("m,n,lda", [(1, 1, 1), (7, 9, 8), (37, 29, 40), (1000, 300, 1001), (2048, 2048, 2048),
                                     (1001, 77, 1004)])
@pytest.mark.parametrize("incs", [(1, 1), (2, 3)])
def test_sger_bit_exact(cuda, m, n, lda, incs):
    incx, incy = incs
    x, y = rnd((m - 1) * incx + 1, 1), rnd((n - 1) * incy + 1, 2)
    y[::incy][: n // 3] = 0.0  # zero coefficients skip the column (sger.rs:93-96)
    a = rnd(lda * n, 3)
    a[5 % a.size] = np.nan
    A = dev(a)
    cb.sger(m, n, 0.75, dev(x), incx, dev(y), incy, A, lda)
    np.testing.assert_array_equal(host(A), oracle.sger(m, n, 0.75, x, incx, y, incy, a, lda))


@pytest.mark.parametrize("n,lda", [(1, 1), (9, 9), (37, 41), (1000, 1000), (37, 40), (1001, 1004)])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("inc", [1, 2])
def test_ssyr_ssyr2_bit_exact(cuda, n, lda, uplo, inc):
    x, y = rnd((n - 1) * inc + 1, 1), rnd((n - 1) * inc + 1, 2)
    x[::inc][1::4] = 0.0
    y[::inc][2::5] = 0.0
    a = rnd(lda * n, 3)
    A = dev(a)
    cb.ssyr(uplo, n, -0.5, dev(x), inc, A, lda)
    np.testing.assert_array_equal(host(A), oracle.ssyr(uplo, n, -0.5, x, inc, a, lda))
    A = dev(a)
    cb.ssyr2(uplo, n, 1.25, dev(x), inc, dev(y), inc, A, lda)
    np.testing.assert_array_equal(host(A), oracle.ssyr2(uplo, n, 1.25, x, inc, y, inc, a, lda))
