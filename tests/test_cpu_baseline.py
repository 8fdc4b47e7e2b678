"""The CPU baseline the reference arm of bench.py times (oracle/oracle.c
port_sgemm_nn, port_sgemv_{n,t}, port_sdot: CORAL's blocking and loop order
restated in C) computes the right results: the reference's own SGEMM / SGEMV
fixtures (BLAS outputs in tests/golden/golden.npz), and a shape that crosses
every MC/NC/KC block edge against the double-double oracle."""
import numpy as np
import pytest

import fixtures as fx
import oracle
from conftest import allclose_ref


@pytest.mark.parametrize("si", range(len(fx.GEMM_SHAPES)))
def test_port_sgemm_nn_fixtures(golden, si):
    m, n, k, lda, _, ldb, _, ldc = fx.GEMM_SHAPES[si]
    a, b, c0 = fx.gemm_operands(0, 0, m, n, k, lda, ldb, ldc)
    for ci, (alpha, beta) in enumerate(fx.GEMM_ALPHA_BETA):
        c = c0.copy()
        oracle.port_sgemm_nn(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
        full = c.reshape(n, ldc).T[:m, :]
        if si < 3:
            allclose_ref(full.ravel(order="F"), golden[f"sgemm_s{si}_00_c{ci}"], 1e-5, 1e-5)
        else:
            ri, cj = fx.sample_positions(m, n, 64)
            # sgemm_tests.rs:85-86
            allclose_ref(full[ri, cj], golden[f"sgemm_big_s{si}_00_c{ci}"], 1e-3, 1e-3)


def test_port_sgemm_nn_crosses_every_block_edge():
    """m > MC (384), n > NC (576), k > KC (256), ragged register tiles and
    padded leading dimensions: component-wise within k fp32 roundings."""
    m, n, k, lda, ldb, ldc = 401, 603, 517, 409, 523, 405
    rng = np.random.default_rng(5)
    a = rng.uniform(-1, 1, lda * k).astype(np.float32)
    b = rng.uniform(-1, 1, ldb * n).astype(np.float32)
    c0 = rng.uniform(-1, 1, ldc * n).astype(np.float32)
    c = c0.copy()
    oracle.port_sgemm_nn(m, n, k, 1.5, a, lda, b, ldb, 0.5, c, ldc)
    ii, jj = rng.integers(0, m, 2048), rng.integers(0, n, 2048)
    want, bound = oracle.gemm_sample(0, 0, m, n, k, 1.5, a, lda, b, ldb, 0.5, c0, ldc, ii, jj)
    got = c[ii + jj * ldc].astype(np.float64)
    assert (np.abs(got - want) <= (k + 2) * 2.0**-24 * bound).all()
    # rows past m of each column are untouched
    pad = np.ones(ldc * n, bool)
    for j in range(n):
        pad[j * ldc:j * ldc + m] = False
    np.testing.assert_array_equal(c[pad], c0[pad])


def test_port_sgemm_nn_scale_only():
    """alpha = 0 or k = 0 scale C by beta (beta = 0 writes zeros),
    sgemm_nn.rs:29-45."""
    c0 = np.arange(12, dtype=np.float32)
    for beta, want in ((0.0, np.zeros(12, np.float32)), (1.0, c0), (0.5, c0 * np.float32(0.5))):
        c = c0.copy()
        oracle.port_sgemm_nn(3, 4, 5, 0.0, np.ones(15, np.float32), 3, np.ones(20, np.float32), 5, beta, c, 3)
        np.testing.assert_array_equal(c, want)
        c = c0.copy()
        oracle.port_sgemm_nn(3, 4, 0, 1.0, np.ones(1, np.float32), 3, np.ones(1, np.float32), 1, beta, c, 3)
        np.testing.assert_array_equal(c, want)


@pytest.mark.parametrize("si", range(len(fx.GEMV_SHAPES)))
def test_port_sgemv_fixtures(golden, si):
    m, n, lda, _ = fx.GEMV_SHAPES[si]
    a = fx.gemv_matrix(m, n, lda)
    for trans in (0, 1):
        xl, yl = (n, m) if trans == 0 else (m, n)
        x, y0 = fx.gemv_x(xl, 1), fx.gemv_y(yl, 1)
        for ci, (alpha, beta) in enumerate(fx.GEMV_COEFFS):
            y = y0.copy()
            oracle.port_sgemv(trans, m, n, alpha, a, lda, x, beta, y)
            # sgemv_tests.rs tolerance 1e-5
            allclose_ref(y, golden[f"sgemv_s{si}_11_t{trans}_c{ci}"], 1e-5, 1e-5)


def test_port_sdot_matches_oracle():
    """dot_tests.rs real n = 1024 ramps, at the file's f32 tolerance 4e-6
    (dot_tests.rs:176-177), and a long random vector."""
    x = fx.strided(1024, 1, lambda k: fx.f32(0.05) + fx.f32(0.03) * k)
    y = fx.strided(1024, 1, lambda k: fx.f32(-0.3) + fx.f32(0.002) * k)
    want = oracle.sdot(1024, x, 1, y, 1)
    assert abs(oracle.port_sdot(1024, x, y) - want) <= 4e-6 + 4e-6 * abs(want)
    rng = np.random.default_rng(9)
    x, y = rng.uniform(-1, 1, (2, 1 << 20)).astype(np.float32)
    want = oracle.sdot(1 << 20, x, 1, y, 1)
    scale = float(np.abs(x.astype(np.float64) * y).sum())
    assert abs(oracle.port_sdot(1 << 20, x, y) - want) <= 64 * 2.0**-24 * scale
