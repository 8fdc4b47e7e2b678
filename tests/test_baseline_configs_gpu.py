"""Parity at the exact sizes of the benchmarked configurations.

The bandwidth and precision figures are measured at these shapes, so each is
also checked here against the oracle, not only at the smaller sizes of the
other parity files:

- plain SGEMM NN, m = n = k = 512, lda = ldb = ldc = 512, alpha = 1.5,
  beta = 0.5, operands U[-1, 1] from a seed: every entry of C against the
  double-double oracle (component-wise bound), plus the reference test's own
  criterion at rtol = atol = 1e-3 (sgemm_tests.rs:85-86);
- SSYMV upper, n = 8192, lda = n, and CHEMV upper, n = 4096, lda = n, with
  NaN in the unstored triangle: all of y at 1e-5 of the scaled bound
  (ssymv_tests.rs:152-153, chemv_tests.rs:190-191);
- SAXPY at n = 2^26, bit for bit against the restatement of saxpy.rs:63-114
  (fused body, rounded tail);
- STRSV lower and upper, N and T, n in {1000, 4096}, on triangles that are
  not diagonally dominant but well posed (diagonal U[1, 2], off-diagonal
  U[-1, 1] / sqrt(n), and four times that), against the substitution-order
  oracle of strlsv.rs:66-140 / strusv.rs at 1e-4 (strsv_tests.rs:213-214).
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle
from conftest import allclose_ref

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


# At k = 512 the error of every mode is set by the fp32 accumulation and the
# final fp32 rounding (up to k * 2^-24 ~ 3e-5 of the bound in the worst case;
# about 1e-6 measured over all 262144 entries for both split modes), so all
# three modes get the native kernel's tolerance.  The 1e-6 bound of the split
# path is checked at 8192^3 in test_gemm_split_gpu.py.
@pytest.mark.parametrize("mode,tol", [(cb.GemmMode.NATIVE, 1e-5), (cb.GemmMode.SPLIT_BF16X3, 1e-5),
                                      (cb.GemmMode.SPLIT_BF16X6, 1e-5)])
def test_sgemm_nn_512_config(cuda, mode, tol):
    n = 512
    rng = np.random.default_rng(512)
    a = rng.uniform(-1, 1, n * n).astype(np.float32)
    b = rng.uniform(-1, 1, n * n).astype(np.float32)
    c = rng.uniform(-1, 1, n * n).astype(np.float32)
    h = cb.handle()
    h.set_gemm_mode(mode)
    try:
        C = dev(c)
        cb.sgemm(0, 0, n, n, n, 1.5, dev(a), n, dev(b), n, 0.5, C, n)
        got = host(C).reshape(n, n).T  # [row, col]
    finally:
        h.set_gemm_mode(cb.GemmMode.NATIVE)
    want, bound = oracle.gemm_full(0, 0, n, n, n, 1.5, a, n, b, n, 0.5, c, n)
    err = np.abs(got - want) / bound
    assert err.max() <= tol, float(err.max())
    allclose_ref(got, want, 1e-3, 1e-3)


def sym_upper(n, seed, complex_=False):
    """Upper triangle stored, NaN below the diagonal; [col][row] flat."""
    rng = np.random.default_rng(seed)
    if complex_:
        a = (rng.uniform(-1, 1, (n, n)) + 1j * rng.uniform(-1, 1, (n, n))).astype(np.complex64)
    else:
        a = rng.uniform(-1, 1, (n, n)).astype(np.float32)
    col, row = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    a[row > col] = np.nan
    return a.reshape(-1)


def abs_sym_matvec(a, n, xabs):
    """(|A_sym|) |x| for an upper-stored matrix, in float64 row blocks."""
    at = np.abs(np.nan_to_num(a.reshape(n, n)))  # [col][row], zeros below the diagonal
    out = np.zeros(n)
    # stored part: sum_j>=i |A(i, j)| |x_j|  -> at.T @ x ; mirror: sum_j<i |A(j, i)| |x_j|
    out += at.T.astype(np.float64) @ xabs
    out += at.astype(np.float64) @ xabs
    out -= np.abs(np.diagonal(at)).astype(np.float64) * xabs
    return out


def test_ssymv_upper_8192_config(cuda):
    n = 8192
    a = sym_upper(n, 8192)
    rng = np.random.default_rng(81)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    y = rng.uniform(-1, 1, n).astype(np.float32)
    Y = dev(y)
    cb.ssymv(0, n, 1.5, dev(a), n, dev(x), 1, 0.5, Y, 1)
    got = host(Y)
    want = oracle.ssymv(0, n, 1.5, a, n, x, 1, 0.5, y, 1)
    assert np.isfinite(got).all()
    scale = 1.5 * abs_sym_matvec(a, n, np.abs(x).astype(np.float64)) + 0.5 * np.abs(y)
    err = np.abs(got - want) / scale
    assert err.max() <= 1e-5, float(err.max())


def test_chemv_upper_4096_config(cuda):
    n = 4096
    a = sym_upper(n, 4096, complex_=True)
    rng = np.random.default_rng(40)
    x = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(np.complex64)
    y = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(np.complex64)
    alpha, beta = (1.5, -0.5), (0.25, 0.0)
    Y = dev(y)
    cb.chemv(0, n, complex(*alpha), dev(a), n, dev(x), 1, complex(*beta), Y, 1)
    got = host(Y)
    w = oracle.chemv(0, n, np.array(alpha, np.float32), a.view(np.float32), n, x.view(np.float32), 1,
                     np.array(beta, np.float32), y.view(np.float32), 1)
    want = w[0::2] + 1j * w[1::2]
    assert np.isfinite(got).all()
    scale = (np.hypot(*alpha) * abs_sym_matvec(np.abs(a), n, np.abs(x).astype(np.float64))
             + np.hypot(*beta) * np.abs(y))
    err = np.abs(got - want) / scale
    assert err.max() <= 1e-5, float(err.max())


def test_saxpy_2p26_bit_exact(cuda):
    n = 1 << 26
    rng = np.random.default_rng(26)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    y = rng.uniform(-1, 1, n).astype(np.float32)
    Y = dev(y)
    cb.saxpy(n, 0.7312, dev(x), 1, Y, 1)
    want = oracle.saxpy(n, 0.7312, x, 1, y, 1)
    got = host(Y)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def ill_triangle(n, uplo, seed, off_scale):
    """Not diagonally dominant, well posed: diag U[1, 2], off-diagonal
    U[-1, 1] * off_scale / sqrt(n); NaN in the unstored triangle."""
    rng = np.random.default_rng(seed)
    a = (rng.uniform(-1, 1, (n, n)) * (off_scale / np.sqrt(n))).astype(np.float32)  # [col][row]
    col, row = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    stored = (row <= col) if uplo == 0 else (row >= col)
    a[~stored] = np.nan
    d = np.arange(n)
    a[d, d] = rng.uniform(1, 2, n).astype(np.float32)
    return a.reshape(-1)


@pytest.mark.parametrize("n", [1000, 4096])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("off_scale", [1.0, 4.0])
def test_strsv_not_dominant(cuda, n, uplo, trans, off_scale):
    a = ill_triangle(n, uplo, n + 7 * uplo + 3 * trans, off_scale)
    b = np.random.default_rng(n + 1).uniform(-1, 1, n).astype(np.float32)
    X = dev(b)
    cb.strsv(uplo, trans, 1, n, dev(a), n, X, 1)
    got = host(X)
    want = oracle.strsv(uplo, trans, 1, n, a, n, b, 1)
    assert np.isfinite(got).all()
    allclose_ref(got, want, 1e-4, 1e-4)
