"""Closed-form operand generators of the reference's own test suite.

Each generator reproduces, in numpy float32 arithmetic, the deterministic
fixture of the cited reference test (no RNG there), so the same inputs can be
rebuilt here, in the GPU tests and in make_golden.py.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def colmajor(rows: int, cols: int, ld: int, f) -> np.ndarray:
    """Flat column-major buffer of ld*cols floats (sgemm_tests.rs:48-62)."""
    a = np.zeros(ld * cols, np.float32)
    i = np.arange(rows, dtype=np.float32)
    for j in range(cols):
        a[j * ld:j * ld + rows] = f(i, f32(j))
    return a


def strided(length: int, inc: int, f) -> np.ndarray:
    """iamax_tests.rs:17-28 / sgemv_tests.rs:65-80 make_strided_vec."""
    v = np.zeros((length - 1) * inc + 1 if length else 1, np.float32)
    k = np.arange(length)
    v[k * inc] = f(k.astype(np.float32)).astype(np.float32)
    return v


# ---- sgemm_tests.rs:112-114 -------------------------------------------------
def gemm_a(i, j):
    return f32(0.1) + i * f32(0.25) + j * f32(0.125)


def gemm_b(i, j):
    return f32(-0.2) + i * f32(0.05) - j * f32(0.075)


def gemm_c(i, j):
    return f32(0.3) - i * f32(0.01) + j * f32(0.02)


GEMM_ALPHA_BETA = [(1.0, 0.0), (0.5, 1.0), (0.75, -0.25), (0.0, 0.7)]   # sgemm_tests.rs:151-156
# (m, n, k, lda_n, lda_t, ldb_n, ldb_t, ldc): sgemm_tests.rs:188-236
GEMM_SHAPES = [
    (5, 7, 4, 5, 4, 4, 7, 5),
    (13, 14, 11, 13, 11, 11, 14, 13),
    (17, 19, 13, 20, 15, 18, 23, 24),
    (128, 128, 128, 128, 128, 128, 128, 128),
    (64, 192, 15, 64, 15, 15, 192, 64),
    (192, 64, 15, 192, 15, 15, 64, 192),
]


def gemm_operands(op_a: int, op_b: int, m, n, k, lda, ldb, ldc):
    a_rows, a_cols = (m, k) if op_a == 0 else (k, m)
    b_rows, b_cols = (k, n) if op_b == 0 else (n, k)
    a = colmajor(a_rows, a_cols, lda, gemm_a)
    b = colmajor(b_rows, b_cols, ldb, gemm_b)
    c = colmajor(m, n, ldc, gemm_c)
    return a, b, c


# ---- sgemv_tests.rs:49-63, 145-155, 205-246 ---------------------------------
def gemv_matrix(m, n, lda):
    return colmajor(m, n, lda, lambda i, j: f32(0.1) + i * f32(0.5) + j * f32(0.25))


GEMV_COEFFS = [(1.0, 0.0), (0.0, -0.75), (0.75, -0.25), (-0.6, 0.4), (1.1, 0.0), (0.85, 0.1)]
# (m, n, lda, [(incx, incy)])
GEMV_SHAPES = [
    (5, 4, 5, [(1, 1)]),
    (1024, 512, 1024, [(1, 1), (2, 3), (3, 2), (2, 1)]),
    (256, 1024, 263, [(1, 1)]),
    (640, 320, 640, [(1, 1)]),
]


def gemv_x(length, inc):
    return strided(length, inc, lambda k: f32(0.2) + f32(0.1) * k)


def gemv_y(length, inc):
    return strided(length, inc, lambda k: f32(-0.3) + f32(0.05) * k)


# ---- strsv_tests.rs:60-118, 300-335 -----------------------------------------
def trsv_matrix(n, lda, uplo):
    """uplo 0: make_upper, 1: make_lower, 2: make_padded (both triangles)."""
    a = np.zeros(lda * n, np.float32)
    for j in range(n):
        for i in range(n):
            if uplo == 0 and i > j:
                continue
            if uplo == 1 and i < j:
                continue
            if i == j:
                a[i + j * lda] = f32(1.0) + f32(0.02) * f32(i)
            else:
                d = f32(abs(i - j))
                a[i + j * lda] = f32(0.01) / (f32(1.0) + d)
    return a


def trsv_x(n, inc):
    return strided(n, inc, lambda k: f32(0.05) + f32(0.01) * k)


# (n, lda, incs)
TRSV_SHAPES = [(7, 7, [1]), (127, 132, [1]), (640, 640, [2, 3]), (1024, 1024, [1])]


# ---- iamax_tests.rs:79-170 ---------------------------------------------------
def isamax_cases():
    """(n, incx, x) of the reference's planted-maximum cases."""
    cases = []
    x = strided(1024, 1, lambda k: np.where(
        k == 777, f32(-1234.5),
        np.abs(np.sin(k) * f32(3.0)) * np.where(k % 2 == 0, f32(1.0), f32(-1.0))))
    cases.append((1024, 1, x))
    x = strided(777, 3, lambda k: np.where(
        k == 321, f32(9999.0),
        (f32(0.2) - f32(0.001) * k) * np.where(k % 2 == 0, f32(1.0), f32(-1.0))))
    cases.append((777, 3, x))
    cases.append((0, 1, np.full(5, 2.0, np.float32)))
    cases.append((1, 5, strided(1, 5, lambda k: np.full_like(k, -3.14159))))
    return cases


# ---- doctests -----------------------------------------------------------------
# coral-aarch64/src/level3/sgemm.rs:36-81 (alpha=2, beta=1, C = I)
SGEMM_DOCTEST = dict(
    a=np.array([1, 2, 3, 4], np.float32), b=np.array([5, 6, 7, 8], np.float32),
    c=np.array([1, 0, 0, 1], np.float32), alpha=2.0, beta=1.0,
    expect=np.array([47, 68, 62, 93], np.float32))
# coral-aarch64/src/level3/cgemm.rs:36-96 (alpha = 2+i, beta = 1-i)
CGEMM_DOCTEST = dict(
    a=np.array([1 + 2j, 5 + 6j, 3 + 4j, 7 + 8j], np.complex64),
    b=np.array([9 + 1j, 4 + 5j, 2 + 3j, 6 + 7j], np.complex64),
    c=np.array([1 + 1j, 3 + 0j, 0 + 2j, 4 + 1j], np.complex64),
    alpha=2 + 1j, beta=1 - 1j,
    expect=np.array([-50 + 99j, -69 + 276j, -78 + 92j, -163 + 223j], np.complex64))
