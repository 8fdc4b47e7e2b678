"""Double and complex rank-1 / rank-2 updates through the C ABI.

DGER, CGERU/CGERC, ZGERU/ZGERC, DSYR, DSYR2, CHER/ZHER, CHER2/ZHER2 against
the oracle (dger.rs, cgeru.rs, cgerc.rs, dsyr.rs, dsyr2.rs, cher.rs,
cher2.rs and the z variants).  Each updated element must match within
tol (|A| + |terms|) (tol 1e-13 for double data, 1e-6 for complex64, where the
reference forms the coefficient in fp32); elements outside the updated
triangle hold NaN and must come back bit for bit; a column whose coefficient
is zero is left untouched (y_j = 0 is planted); Hermitian updates leave a real
diagonal.
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle

pytestmark = pytest.mark.gpu
TOL = {"d": 1e-13, "c": 1e-6, "z": 1e-13}
DT = {"d": np.float64, "c": np.complex64, "z": np.complex128}


def rnd(rng, shape, kind):
    dt = DT[kind]
    if kind == "d":
        return rng.uniform(-1, 1, shape).astype(dt)
    return (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(dt)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def check(got, want, a0, terms, kind):
    fin = np.isfinite(want)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(want))
    scale = np.abs(a0[fin]) + terms[fin]
    assert (np.abs(got[fin] - want[fin]) <= TOL[kind] * scale + 1e-30).all(), np.abs(got[fin] - want[fin]).max()


@pytest.mark.parametrize("kind,conj", [("d", 0), ("c", 0), ("c", 1), ("z", 0), ("z", 1)])
@pytest.mark.parametrize("m,n,lda,inc", [(1, 1, 1, 1), (300, 211, 305, 1), (1500, 1100, 1500, 1), (257, 129, 260, 3),
                                          (301, 211, 304, 1), (33, 17, 36, 1)])
def test_ger(cuda, kind, conj, m, n, lda, inc):
    rng = np.random.default_rng(m + n + conj)
    a = rnd(rng, (n, lda), kind)
    a[:, m:] = np.nan                                  # rows past m: never touched
    x = rnd(rng, (m - 1) * inc + 1, kind)
    y = rnd(rng, (n - 1) * inc + 1, kind)
    y[0] = 0                                            # column 0: zero coefficient, untouched
    alpha = 0.75 if kind == "d" else 0.75 - 0.5j
    A = dev(a.ravel())
    if kind == "d":
        cb.dger(m, n, alpha, dev(x), inc, dev(y), inc, A, lda)
        want = oracle.dger(m, n, alpha, x, inc, y, inc, a.ravel(), lda)
    else:
        fn = {("c", 0): cb.cgeru, ("c", 1): cb.cgerc, ("z", 0): cb.zgeru, ("z", 1): cb.zgerc}[(kind, conj)]
        fn(m, n, alpha, dev(x), inc, dev(y), inc, A, lda)
        want = oracle.gerc_u(kind, conj, m, n, alpha, x, inc, y, inc, a.ravel(), lda)
    torch.cuda.synchronize()
    got = A.cpu().numpy()
    terms = abs(alpha) * np.outer(np.abs(y[::inc][:n]), np.pad(np.abs(x[::inc][:m]), (0, lda - m))).ravel()
    check(got.astype(np.complex128), want.astype(np.complex128), a.ravel().astype(np.complex128), terms, kind)
    np.testing.assert_array_equal(got.reshape(n, lda)[0], a[0])   # zero-coefficient column


@pytest.mark.parametrize("kind,two", [("d", 0), ("d", 1), ("c", 0), ("c", 1), ("z", 0), ("z", 1)])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("n,lda,inc", [(1, 1, 1), (7, 9, 1), (300, 300, 1), (1030, 1035, 1), (129, 130, 2),
                                       (1031, 1032, 1), (13, 16, 1)])
def test_syr_her(cuda, kind, two, uplo, n, lda, inc):
    rng = np.random.default_rng(n * 3 + uplo + 7 * two)
    a = rnd(rng, (n, lda), kind)
    jj, ii = np.meshgrid(np.arange(n), np.arange(lda), indexing="ij")
    stored = (ii <= jj) if uplo == 0 else (ii >= jj)
    a[~stored] = np.nan                                 # outside the triangle (and past n): untouched
    x = rnd(rng, (n - 1) * inc + 1, kind)
    y = rnd(rng, (n - 1) * inc + 1, kind) if two else None
    alpha = 0.6 if (kind == "d" or not two) else 0.6 - 0.4j
    A = dev(a.ravel())
    if kind == "d":
        if two:
            cb.dsyr2(uplo, n, alpha, dev(x), inc, dev(y), inc, A, lda)
        else:
            cb.dsyr(uplo, n, alpha, dev(x), inc, A, lda)
        want = oracle.dsyr(uplo, n, alpha, x, inc, a.ravel(), lda, y=y, incy=inc)
    else:
        if two:
            fn = cb.cher2 if kind == "c" else cb.zher2
            fn(uplo, n, alpha, dev(x), inc, dev(y), inc, A, lda)
        else:
            fn = cb.cher if kind == "c" else cb.zher
            fn(uplo, n, alpha, dev(x), inc, A, lda)
        want = oracle.her(kind, uplo, n, alpha, x, inc, a.ravel(), lda, y=y, incy=inc)
    torch.cuda.synchronize()
    got = A.cpu().numpy()
    xa = np.pad(np.abs(x[::inc][:n]), (0, lda - n))
    ya = np.pad(np.abs(y[::inc][:n]), (0, lda - n)) if two else xa
    terms = (abs(alpha) * (np.outer(np.abs(ya[:n]), xa) + np.outer(np.abs(xa[:n]), ya))).ravel()
    check(got.astype(np.complex128), want.astype(np.complex128), a.ravel().astype(np.complex128), terms, kind)
    if kind != "d":
        d = np.arange(n)
        assert (got.reshape(n, lda)[d, d].imag == 0).all()  # Hermitian: real diagonal
