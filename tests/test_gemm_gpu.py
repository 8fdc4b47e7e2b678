"""Level-3 parity through the C ABI (coral-aarch64/src/level3).

Native-precision paths: the reference's own fixture cases against golden
CBLAS outputs with its tolerance (tests/level3/sgemm_tests.rs:85-86), the
doctests exactly, and seeded random operands against the double-double oracle
with a component-wise bound |C - C_oracle| <= tol * (|alpha| |op(A)||op(B)| +
|beta||C|): tol = 1e-5 (fp32: k * 2^-24 for k <= 128 plus margin), 1e-13 (fp64).
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


def test_sgemm_doctest(cuda):
    d = fx.SGEMM_DOCTEST
    C = dev(d["c"])
    cb.sgemm(0, 0, 2, 2, 2, d["alpha"], dev(d["a"]), 2, dev(d["b"]), 2, d["beta"], C, 2)
    np.testing.assert_array_equal(host(C), d["expect"])


def test_cgemm_doctest(cuda):
    d = fx.CGEMM_DOCTEST
    C = dev(d["c"])
    cb.cgemm(0, 0, 2, 2, 2, d["alpha"], dev(d["a"]), 2, dev(d["b"]), 2, d["beta"], C, 2)
    np.testing.assert_array_equal(host(C), d["expect"])


@pytest.mark.parametrize("si", range(3))
def test_sgemm_reference_fixtures(cuda, golden, si):
    m, n, k, lda_n, lda_t, ldb_n, ldb_t, ldc = fx.GEMM_SHAPES[si]
    for (op_a, op_b) in [(0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (0, 2)]:
        lda = lda_n if op_a == 0 else lda_t
        ldb = ldb_n if op_b == 0 else ldb_t
        a, b, c = fx.gemm_operands(op_a, op_b, m, n, k, lda, ldb, ldc)
        for ci, (alpha, beta) in enumerate(fx.GEMM_ALPHA_BETA):
            C = dev(c)
            cb.sgemm(op_a, op_b, m, n, k, alpha, dev(a), lda, dev(b), ldb, beta, C, ldc)
            got = host(C).reshape(n, ldc).T
            allclose_ref(got[:m, :].ravel(order="F"), golden[f"sgemm_s{si}_{op_a}{op_b}_c{ci}"],
                         1e-3, 1e-3)
            np.testing.assert_array_equal(got[m:, :], c.reshape(n, ldc).T[m:, :])  # ld padding untouched


@pytest.mark.parametrize("si", [3, 4, 5])
def test_sgemm_reference_shapes_vs_oracle(cuda, si):
    m, n, k, lda_n, lda_t, ldb_n, ldb_t, ldc = fx.GEMM_SHAPES[si]
    for (op_a, op_b) in [(0, 0), (0, 1), (1, 0), (1, 1)]:
        lda = lda_n if op_a == 0 else lda_t
        ldb = ldb_n if op_b == 0 else ldb_t
        a, b, c = fx.gemm_operands(op_a, op_b, m, n, k, lda, ldb, ldc)
        for alpha, beta in fx.GEMM_ALPHA_BETA:
            C = dev(c)
            cb.sgemm(op_a, op_b, m, n, k, alpha, dev(a), lda, dev(b), ldb, beta, C, ldc)
            want, _ = oracle.gemm_full(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
            allclose_ref(host(C).reshape(n, ldc).T[:m, :], want, 1e-3, 1e-3)


def rnd(shape, seed, dtype):
    rng = np.random.default_rng(seed)
    if np.issubdtype(dtype, np.complexfloating):
        return (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(dtype)
    return rng.uniform(-1, 1, shape).astype(dtype)


def gemm_case(fn, dtype, op_a, op_b, m, n, k, alpha, beta, tol, pad=3, seed=0, sample=None):
    lda = (m if op_a == 0 else k) + pad
    ldb = (k if op_b == 0 else n) + pad
    ldc = m + pad
    a = rnd(lda * (k if op_a == 0 else m), seed, dtype)
    b = rnd(ldb * (n if op_b == 0 else k), seed + 1, dtype)
    c = rnd(ldc * n, seed + 2, dtype)
    C = dev(c)
    fn(op_a, op_b, m, n, k, alpha, dev(a), lda, dev(b), ldb, beta, C, ldc)
    got = host(C).reshape(n, ldc).T
    if sample is None:
        ii, jj = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
        ii, jj = ii.ravel(), jj.ravel()
    else:
        rng = np.random.default_rng(seed + 3)
        ii, jj = rng.integers(0, m, sample), rng.integers(0, n, sample)
    want, bound = oracle.gemm_sample(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ii, jj)
    err = np.abs(got[ii, jj].astype(np.complex128 if np.iscomplexobj(got) else np.float64) - want)
    worst = float((err / np.maximum(bound, 1e-300)).max()) if err.size else 0.0
    assert worst <= tol, worst
    np.testing.assert_array_equal(got[m:, :], c.reshape(n, ldc).T[m:, :])
    return worst


SHAPES = [(1, 1, 1), (5, 7, 4), (127, 129, 65), (256, 256, 256), (300, 77, 513)]
OPS_REAL = [(0, 0), (0, 1), (1, 0), (1, 1), (2, 2)]
OPS_CPLX = [(a, b) for a in (0, 1, 2) for b in (0, 1, 2)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("ops", OPS_REAL)
def test_sgemm_native_random(cuda, shape, ops):
    m, n, k = shape
    for alpha, beta in [(1.5, 0.5), (1.0, 0.0), (-0.3, 1.0)]:
        gemm_case(cb.sgemm, np.float32, *ops, m, n, k, alpha, beta, 1e-5)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("ops", OPS_REAL)
def test_dgemm_native_random(cuda, shape, ops):
    m, n, k = shape
    for alpha, beta in [(1.5, 0.5), (1.0, 0.0)]:
        gemm_case(cb.dgemm, np.float64, *ops, m, n, k, alpha, beta, 1e-13)


@pytest.mark.parametrize("shape", SHAPES[:4])
@pytest.mark.parametrize("ops", OPS_CPLX)
def test_cgemm_native_random(cuda, shape, ops):
    m, n, k = shape
    gemm_case(cb.cgemm, np.complex64, *ops, m, n, k, 1.5 - 0.5j, 0.25 + 1j, 2e-5)
    gemm_case(cb.cgemm, np.complex64, *ops, m, n, k, 1.0, 0.0, 2e-5)


@pytest.mark.parametrize("shape", SHAPES[:4])
@pytest.mark.parametrize("ops", OPS_CPLX)
def test_zgemm_native_random(cuda, shape, ops):
    m, n, k = shape
    gemm_case(cb.zgemm, np.complex128, *ops, m, n, k, 1.5 - 0.5j, 0.25 + 1j, 1e-13)


def test_gemm_scale_only_paths(cuda):
    m, n = 33, 17
    c = rnd(m * n, 5, np.float32)
    for alpha, k, beta in [(0.0, 8, 0.5), (1.0, 0, 0.5), (0.0, 8, 0.0), (0.0, 8, 1.0)]:
        C = dev(c)
        a = dev(rnd(m * max(k, 1), 6, np.float32))
        b = dev(rnd(max(k, 1) * n, 7, np.float32))
        cb.sgemm(0, 0, m, n, k, alpha, a, m, b, max(k, 1), beta, C, m)
        want = np.zeros_like(c) if beta == 0.0 else (c * np.float32(beta) if beta != 1.0 else c)
        np.testing.assert_array_equal(host(C), want)


def test_gemm_bad_args(cuda):
    A = dev(np.zeros(64, np.float32))
    with pytest.raises(cb.CoralError) as e:
        cb.sgemm(0, 0, 8, 8, 8, 1.0, A, 7, A, 8, 0.0, A, 8)
    assert e.value.bad_arg == 8
    with pytest.raises(cb.CoralError) as e:
        cb.sgemm(0, 0, 8, 8, 8, 1.0, A, 8, A, 8, 0.0, A, 4)
    assert e.value.bad_arg == 13


def test_sgemm_8192_sampled(cuda):
    """The 8192^3 precision-set shape in plain FP32, checked on sampled entries."""
    m = n = k = 8192
    rng = np.random.default_rng(1)
    A = torch.empty(m * k, dtype=torch.float32, device="cuda").uniform_(-1, 1)
    B = torch.empty(k * n, dtype=torch.float32, device="cuda").uniform_(-1, 1)
    Cm = torch.empty(m * n, dtype=torch.float32, device="cuda").uniform_(-1, 1)
    a, b, c = A.cpu().numpy(), B.cpu().numpy(), Cm.cpu().numpy()
    cb.sgemm(0, 0, m, n, k, 1.5, A, m, B, k, 0.5, Cm, m)
    got = host(Cm)
    ii, jj = rng.integers(0, m, 512), rng.integers(0, n, 512)
    want, bound = oracle.gemm_sample(0, 0, m, n, k, 1.5, a, m, b, k, 0.5, c, m, ii, jj)
    err = np.abs(got[ii + jj * m] - want)
    assert float((err / bound).max()) <= 1e-5
