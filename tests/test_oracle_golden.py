"""Pins the CPU oracle against the reference's known answers and fixtures.

Known answers: the sgemm and cgemm doctests (coral-aarch64/src/level3/
sgemm.rs:36-81, cgemm.rs:36-96) and the planted-maximum isamax cases
(tests/level1/iamax_tests.rs:79-170).  Fixtures: the closed-form cases of
tests/level3/sgemm_tests.rs, tests/level2/sgemv_tests.rs and
tests/level2/strsv_tests.rs, whose expected outputs were computed by
CBLAS-class BLAS (tests/golden/make_golden.py) and are checked here with the
reference's own tolerances.
"""
import numpy as np
import pytest

import fixtures as fx
import oracle


def test_sgemm_doctest():
    d = fx.SGEMM_DOCTEST
    vals, _ = oracle.gemm_full(0, 0, 2, 2, 2, d["alpha"], d["a"], 2, d["b"], 2, d["beta"], d["c"], 2)
    np.testing.assert_array_equal(vals.ravel(order="F"), d["expect"])


def test_cgemm_doctest():
    d = fx.CGEMM_DOCTEST
    vals, _ = oracle.gemm_full(0, 0, 2, 2, 2, d["alpha"], d["a"], 2, d["b"], 2, d["beta"], d["c"], 2)
    np.testing.assert_array_equal(vals.ravel(order="F"), d["expect"])


def test_isamax_planted(golden):
    for ci, (n, inc, x) in enumerate(fx.isamax_cases()):
        assert oracle.isamax(n, x, inc) == int(golden[f"isamax_c{ci}"][0])


def test_isamax_nan_and_ties():
    x = np.array([np.nan, -3.0, 3.0, np.nan, -3.0], np.float32)
    assert oracle.isamax(5, x, 1) == 1
    assert oracle.isamax(3, np.full(3, np.nan, np.float32), 1) == 0
    assert oracle.isamax(4, np.zeros(4, np.float32), 1) == 0


@pytest.mark.parametrize("si", range(3))
def test_sgemm_fixtures(golden, si):
    m, n, k, lda_n, lda_t, ldb_n, ldb_t, ldc = fx.GEMM_SHAPES[si]
    for (op_a, op_b) in [(0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (0, 2)]:
        lda = lda_n if op_a == 0 else lda_t
        ldb = ldb_n if op_b == 0 else ldb_t
        a, b, c = fx.gemm_operands(op_a, op_b, m, n, k, lda, ldb, ldc)
        for ci, (alpha, beta) in enumerate(fx.GEMM_ALPHA_BETA):
            vals, _ = oracle.gemm_full(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
            want = golden[f"sgemm_s{si}_{op_a}{op_b}_c{ci}"]
            # sgemm_tests.rs:85-86 (RTOL = ATOL = 1e-3); fp64 vs OpenBLAS fp32 agrees far closer
            from conftest import allclose_ref
            allclose_ref(vals.ravel(order="F"), want, 1e-5, 1e-5)


def test_sgemv_fixtures(golden):
    from conftest import allclose_ref
    for si, (m, n, lda, strides) in enumerate(fx.GEMV_SHAPES):
        a = fx.gemv_matrix(m, n, lda)
        for (incx, incy) in strides:
            for trans in (0, 1):
                xl, yl = (n, m) if trans == 0 else (m, n)
                x = fx.gemv_x(xl, incx)
                y0 = fx.gemv_y(yl, incy)
                for ci, (alpha, beta) in enumerate(fx.GEMV_COEFFS):
                    got = oracle.sgemv(trans, m, n, alpha, a, lda, x, incx, beta, y0, incy)
                    # sgemv_tests.rs:116-117 tolerance 1e-5 (relative to the large sums)
                    allclose_ref(got, golden[f"sgemv_s{si}_{incx}{incy}_t{trans}_c{ci}"], 1e-5, 1e-5)


def test_strsv_fixtures(golden):
    from conftest import allclose_ref
    for si, (n, lda, incs) in enumerate(fx.TRSV_SHAPES):
        for uplo in (0, 1):
            a = fx.trsv_matrix(n, lda, uplo)
            for inc in incs:
                x = fx.trsv_x(n, inc)
                for trans in (0, 1):
                    for diag in (0, 1):
                        got = oracle.strsv(uplo, trans, diag, n, a, lda, x, inc)
                        # strsv_tests.rs:213-214 tolerance 1e-4
                        allclose_ref(got, golden[f"strsv_s{si}_u{uplo}_i{inc}_t{trans}_d{diag}"],
                                     1e-4, 1e-4)


def test_strsv_padded_triangle_ignored():
    """strsv_tests.rs:337-360: the unreferenced triangle (populated) is ignored."""
    n, lda = 127, 132
    full = fx.trsv_matrix(n, lda, 2)
    low = fx.trsv_matrix(n, lda, 1)
    x = fx.trsv_x(n, 1)
    for trans in (0, 1):
        np.testing.assert_array_equal(oracle.strsv(1, trans, 1, n, full, lda, x, 1),
                                      oracle.strsv(1, trans, 1, n, low, lda, x, 1))


def test_level1_against_numpy():
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, 1001).astype(np.float32)
    y = rng.uniform(-1, 1, 1001).astype(np.float32)
    assert abs(oracle.sdot(1001, x, 1, y, 1) - float(np.dot(x.astype(np.float64), y))) < 1e-12
    assert abs(oracle.snrm2(1001, x, 1) - float(np.linalg.norm(x.astype(np.float64)))) < 1e-12
    assert oracle.snrm2(0, x, 1) == 0.0 and oracle.snrm2(5, x, 0) == 0.0
    # saxpy: fused body (first n - n%8), two-rounding tail
    r = oracle.saxpy(1001, 0.3, x, 1, y, 1)
    n8 = 1000
    body = (np.float64(np.float32(0.3)) * x[:n8].astype(np.float64) + y[:n8]).astype(np.float32)
    tail = (np.float32(0.3) * x[n8:]) + y[n8:]
    np.testing.assert_array_equal(r[:n8], body)
    np.testing.assert_array_equal(r[n8:], tail)
    rs = oracle.saxpy(500, 0.3, x, 2, y, 2)
    np.testing.assert_array_equal(rs[::2][:500], (np.float32(0.3) * x[::2][:500]) + y[::2][:500])


def test_rank_updates_reference_rounding():
    rng = np.random.default_rng(3)
    m, n, lda = 37, 29, 40
    x = rng.uniform(-1, 1, m).astype(np.float32)
    y = rng.uniform(-1, 1, n).astype(np.float32)
    a = rng.uniform(-1, 1, lda * n).astype(np.float32)
    got = oracle.sger(m, n, 0.7, x, 1, y, 1, a, lda)
    want = a.copy()
    for j in range(n):
        coeff = np.float32(0.7) * y[j]
        col = want[j * lda:j * lda + m]
        nf = m - m % 8
        col[:nf] = (np.float64(coeff) * x[:nf] + col[:nf]).astype(np.float32)
        col[nf:] = col[nf:] + coeff * x[nf:]
    np.testing.assert_array_equal(got, want)


def test_gemm_sample_scale_only():
    c = np.arange(6, dtype=np.float32)
    vals, absb = oracle.gemm_sample(0, 0, 2, 3, 0, 1.0, np.zeros(1, np.float32), 2,
                                    np.zeros(1, np.float32), 1, 0.5, c, 2, [0, 1], [2, 2])
    np.testing.assert_array_equal(vals, [2.0, 2.5])
