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


# ---- double and complex level 1 (coral-aarch64/tests/level1/*.rs) -------------
# Every vector there is a linear ramp a + b k (complex: (a + b k, c + d k)),
# sometimes with alternating signs and one planted element; the generators
# below rebuild them in the element precision.  Each case names its source.
_DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}


def ramp(kind: str, n: int, inc: int, g, alt: bool = False, plant=None) -> np.ndarray:
    """Strided vector of n ramp elements (make_strided_vec / make_strided_cvec)."""
    dt = _DT[kind]
    real = np.float32 if kind in "sc" else np.float64
    v = np.zeros((n - 1) * inc + 1 if n else 1, dt)
    if n == 0:
        return v
    k = np.arange(n).astype(real)
    re = real(g[0]) + real(g[1]) * k
    val = re if kind in "sd" else re + 1j * (real(g[2]) + real(g[3]) * k)
    if alt:
        val = np.where(np.arange(n) % 2 == 0, val, -val)
    val = val.astype(dt)
    if plant is not None:
        val[plant[0]] = plant[1]
    v[np.arange(n) * inc] = val
    return v


L1_CASES = [
    # axpy_tests.rs
    dict(fn="axpy", kind="d", n=1536, incx=1, incy=1, alpha=-2.5, x=(0.25, 0.125), y=(-0.75, 0.05),
         src="axpy_tests.rs:216-226"),
    dict(fn="axpy", kind="d", n=1023, incx=4, incy=3, alpha=0.333333333333, x=(1.0, -1e-3), y=(-0.5, 2e-3),
         src="axpy_tests.rs:252-264"),
    dict(fn="axpy", kind="c", n=800, incx=1, incy=1, alpha=0.75 - 0.2j, x=(0.1, 0.01, -0.05, 0.002),
         y=(-0.2, 0.001, 0.3, -0.003), src="axpy_tests.rs:321-331"),
    dict(fn="axpy", kind="c", n=513, incx=2, incy=3, alpha=-1.1 + 0.4j, x=(0.0, 0.02, 0.03, -0.001),
         y=(0.0, -0.01, 0.04, 0.002), src="axpy_tests.rs:357-369"),
    dict(fn="axpy", kind="c", n=300, incx=1, incy=1, alpha=1j, x=(0.1, 0.001, -0.2, 0.002),
         y=(-0.05, 0.0015, 0.03, -0.001), src="axpy_tests.rs:431-441"),
    dict(fn="axpy", kind="z", n=640, incx=1, incy=1, alpha=1.25 - 0.75j, x=(0.05, 0.002, 0.1, -0.001),
         y=(-0.2, 0.0005, 0.3, 0.0003), src="axpy_tests.rs:468-478"),
    dict(fn="axpy", kind="z", n=511, incx=3, incy=2, alpha=-0.2 + 0.9j, x=(0.0, 0.001, 0.0, -0.002),
         y=(0.4, -0.003, -0.1, 0.004), src="axpy_tests.rs:504-516"),
    dict(fn="axpy", kind="z", n=333, incx=1, incy=1, alpha=2.0, x=(0.3, -0.001, 0.25, 0.002),
         y=(-0.15, 0.0005, 0.07, -0.0003), src="axpy_tests.rs:578-588"),
    # scal_tests.rs (csscal / zdscal reuse the complex ramps with a real alpha)
    dict(fn="scal", kind="d", n=1536, incx=1, alpha=-2.5, x=(0.25, 0.125), src="scal_tests.rs:261-266"),
    dict(fn="scal", kind="d", n=1023, incx=4, alpha=1.0 / 3.0, x=(1.0, -1e-3), src="scal_tests.rs:291-297"),
    dict(fn="scal", kind="d", n=512, incx=1, alpha=0.0, x=(0.2, -0.02), src="scal_tests.rs:322-327"),
    dict(fn="scal", kind="c", n=800, incx=1, alpha=0.75 - 0.2j, x=(0.1, 0.01, -0.05, 0.002),
         src="scal_tests.rs:411-416"),
    dict(fn="scal", kind="c", n=513, incx=3, alpha=-1.1 + 0.4j, x=(0.0, 0.02, 0.03, -0.001),
         src="scal_tests.rs:441-447"),
    dict(fn="scal", kind="c", n=300, incx=1, alpha=1j, x=(0.1, 0.001, -0.2, 0.002), src="scal_tests.rs:532-537"),
    dict(fn="scal", kind="z", n=640, incx=1, alpha=1.25 - 0.75j, x=(0.05, 0.002, 0.1, -0.001),
         src="scal_tests.rs:592-597"),
    dict(fn="scal", kind="z", n=511, incx=2, alpha=-0.2 + 0.9j, x=(0.0, 0.001, 0.0, -0.002),
         src="scal_tests.rs:622-628"),
    dict(fn="scal", kind="z", n=333, incx=1, alpha=2.0, x=(-0.15, 0.0005, 0.07, -0.0003), src="scal_tests.rs:683-688"),
    dict(fn="sscal_r", kind="c", n=513, incx=3, alpha=-1.1, x=(0.0, 0.02, 0.03, -0.001), src="scal_tests.rs:441-447"),
    dict(fn="sscal_r", kind="z", n=640, incx=1, alpha=1.25, x=(0.05, 0.002, 0.1, -0.001), src="scal_tests.rs:592-597"),
    # dot_tests.rs
    dict(fn="dotu", kind="d", n=1536, incx=1, incy=1, x=(0.25, 0.125), y=(-0.75, 0.05), src="dot_tests.rs:305-314"),
    dict(fn="dotu", kind="d", n=1023, incx=4, incy=3, x=(1.0, -1e-3), xalt=True, y=(-0.5, 2e-3),
         src="dot_tests.rs:336-347"),
    dict(fn="dotu", kind="c", n=800, incx=1, incy=1, x=(0.1, 0.01, -0.05, 0.002), y=(-0.2, 0.001, 0.3, -0.003),
         src="dot_tests.rs:429-438"),
    dict(fn="dotu", kind="c", n=513, incx=2, incy=3, x=(0.0, 0.02, 0.03, -0.001), y=(0.0, -0.01, 0.04, 0.002),
         src="dot_tests.rs:462-473"),
    dict(fn="dotc", kind="c", n=800, incx=1, incy=1, x=(0.1, 0.01, -0.05, 0.002), y=(-0.2, 0.001, 0.3, -0.003),
         src="dot_tests.rs:566-575"),
    dict(fn="dotc", kind="c", n=513, incx=2, incy=3, x=(0.0, 0.02, 0.03, -0.001), y=(0.0, -0.01, 0.04, 0.002),
         src="dot_tests.rs:599-610"),
    dict(fn="dotu", kind="z", n=640, incx=1, incy=1, x=(0.05, 0.002, 0.1, -0.001), y=(-0.2, 0.0005, 0.3, 0.0003),
         src="dot_tests.rs:635-644"),
    dict(fn="dotc", kind="z", n=511, incx=3, incy=2, x=(0.0, 0.001, 0.0, -0.002), y=(0.4, -0.003, -0.1, 0.004),
         src="dot_tests.rs:668-674"),
    # asum_tests.rs
    dict(fn="asum", kind="s", n=1024, incx=1, x=(0.05, 0.03), xalt=True, src="asum_tests.rs:114-118"),
    dict(fn="asum", kind="d", n=1536, incx=1, x=(0.25, 0.125), xalt=True, src="asum_tests.rs:217-221"),
    dict(fn="asum", kind="d", n=1023, incx=4, x=(1.0, -1e-3), xalt=True, src="asum_tests.rs:243-248"),
    dict(fn="asum", kind="c", n=800, incx=1, x=(0.1, 0.01, -0.05, 0.002), xalt=True, src="asum_tests.rs:323-330"),
    dict(fn="asum", kind="c", n=513, incx=2, x=(0.0, 0.02, 0.03, -0.001), xalt=True, src="asum_tests.rs:353-361"),
    dict(fn="asum", kind="z", n=640, incx=1, x=(0.05, 0.002, 0.1, -0.001), xalt=True, src="asum_tests.rs:438-445"),
    dict(fn="asum", kind="z", n=511, incx=3, x=(0.0, 0.001, 0.0, -0.002), xalt=True, src="asum_tests.rs:468-476"),
    # nrm2_tests.rs
    dict(fn="nrm2", kind="d", n=1536, incx=1, x=(0.25, 0.125), src="nrm2_tests.rs:205-209"),
    dict(fn="nrm2", kind="d", n=1023, incx=4, x=(1.0, -1e-3), xalt=True, src="nrm2_tests.rs:228-233"),
    dict(fn="nrm2", kind="c", n=800, incx=1, x=(0.1, 0.01, -0.05, 0.002), src="nrm2_tests.rs:299-305"),
    dict(fn="nrm2", kind="c", n=513, incx=2, x=(0.0, 0.02, 0.03, -0.001), src="nrm2_tests.rs:326-333"),
    dict(fn="nrm2", kind="z", n=640, incx=1, x=(0.05, 0.002, 0.1, -0.001), src="nrm2_tests.rs:402-408"),
    dict(fn="nrm2", kind="z", n=511, incx=3, x=(0.0, 0.001, 0.0, -0.002), src="nrm2_tests.rs:429-436"),
    # iamax_tests.rs
    dict(fn="iamax", kind="d", n=1023, incx=4, x=(1.0, -1e-3), xalt=True, src="iamax_tests.rs:207-215"),
    dict(fn="iamax", kind="c", n=800, incx=1, x=(0.1, 0.01, -0.05, 0.002), xalt=True, plant=(400, 999 - 999j),
         src="iamax_tests.rs:282-295"),
    dict(fn="iamax", kind="c", n=513, incx=2, x=(0.0, 0.02, 0.03, -0.001), xalt=True, src="iamax_tests.rs:313-325"),
    dict(fn="iamax", kind="z", n=640, incx=1, x=(0.05, 0.002, 0.1, -0.001), xalt=True, plant=(333, 7777 - 8888j),
         src="iamax_tests.rs:393-405"),
    dict(fn="iamax", kind="z", n=511, incx=3, x=(0.0, 0.001, 0.0, -0.002), xalt=True, src="iamax_tests.rs:424-436"),
    # rot_tests.rs (csrot / zdrot reuse the complex ramps)
    dict(fn="rot", kind="s", n=1024, incx=1, incy=1, theta=0.375, x=(0.05, 0.03), y=(-0.3, 0.002),
         src="rot_tests.rs:86-101"),
    dict(fn="rot", kind="s", n=777, incx=3, incy=2, theta=-0.91, x=(0.2, -0.001), y=(-0.3, 0.002),
         src="rot_tests.rs:135-150"),
    dict(fn="rot", kind="d", n=1536, incx=1, incy=1, theta=0.22, x=(0.25, 0.125), y=(-0.75, 0.05),
         src="rot_tests.rs:271-284"),
    dict(fn="rot", kind="d", n=1023, incx=4, incy=3, theta=-0.61, x=(1.0, -1e-3), y=(-0.5, 2e-3),
         src="rot_tests.rs:318-333"),
    dict(fn="rot", kind="c", n=801, incx=1, incy=1, theta=0.375, x=(0.1, 0.01, -0.05, 0.002),
         y=(-0.2, 0.001, 0.3, -0.003), src="dot_tests.rs:429-438 ramps"),
    dict(fn="rot", kind="z", n=511, incx=3, incy=2, theta=-0.61, x=(0.0, 0.001, 0.0, -0.002),
         y=(0.4, -0.003, -0.1, 0.004), src="dot_tests.rs:668-674 ramps"),
    dict(fn="rotm", kind="s", n=320, incx=1, incy=1, param=(-1.0, 1.1, -0.4, 0.7, 0.9), x=(-0.5, 0.03),
         y=(0.1, 0.002), src="rot_tests.rs:761-772"),
    dict(fn="rotm", kind="s", n=300, incx=1, incy=1, param=(0.0, 0.0, -0.6, 0.8, 0.0), x=(0.2, -0.001),
         y=(-0.3, 0.002), src="rot_tests.rs:804-815"),
    dict(fn="rotm", kind="s", n=300, incx=1, incy=1, param=(1.0, 1.2, 0.0, 0.0, -0.75), x=(0.0, 0.01),
         y=(1.0, -0.005), src="rot_tests.rs:847-858"),
    dict(fn="rotm", kind="s", n=257, incx=2, incy=3, param=(-1.0, -0.3, 0.5, -0.9, 0.4), x=(0.05, 0.01),
         y=(-0.2, 0.003), src="rot_tests.rs:890-903"),
    dict(fn="rotm", kind="d", n=320, incx=1, incy=1, param=(-1.0, 1.05, -0.6, 0.8, 0.95), x=(-1.0, 0.1),
         y=(0.2, 0.004), src="rot_tests.rs:1052-1063"),
    dict(fn="rotm", kind="d", n=300, incx=1, incy=1, param=(0.0, 0.0, -0.25, 0.33, 0.0), x=(1.0, -1e-3),
         y=(-0.5, 2e-3), src="rot_tests.rs:1095-1106"),
    dict(fn="rotm", kind="d", n=300, incx=1, incy=1, param=(1.0, 0.75, 0.0, 0.0, -1.2), x=(0.25, 0.125),
         y=(-0.75, 0.05), src="rot_tests.rs:1138-1149"),
    dict(fn="rotm", kind="d", n=257, incx=2, incy=3, param=(-1.0, -0.8, 0.2, -0.1, 1.3), x=(0.25, 0.125),
         y=(-0.75, 0.05), src="rot_tests.rs:1181-1194"),
]

# The f32 cases of the level-1 files' `real` tests, checked against the oracle
# only (golden keys l1s_c<i>).
L1_S_CASES = [
    dict(fn="axpy", kind="s", n=1024, incx=1, incy=1, alpha=3.1415926, x=(0.05, 0.03), y=(0.10, 0.06),
         src="axpy_tests.rs real, n = 1024"),
    dict(fn="axpy", kind="s", n=777, incx=3, incy=2, alpha=-0.75, x=(0.2, -0.001), y=(-0.3, 0.002),
         src="axpy_tests.rs real, n = 777 strided"),
    dict(fn="axpy", kind="s", n=0, incx=1, incy=1, alpha=1.23, x=(0.0, 0.0), y=(0.0, 0.0),
         src="axpy_tests.rs real, n = 0"),
    dict(fn="scal", kind="s", n=1024, incx=1, alpha=3.1415926, x=(0.05, 0.03), src="scal_tests.rs real, n = 1024"),
    dict(fn="scal", kind="s", n=777, incx=3, alpha=-0.75, x=(0.2, -0.001), src="scal_tests.rs real, n = 777"),
    dict(fn="scal", kind="s", n=4096, incx=1, alpha=0.0, x=(-0.2, 0.001), src="scal_tests.rs real, alpha = 0"),
    dict(fn="scal", kind="s", n=257, incx=1, alpha=1.0, x=(-0.3, 0.01), src="scal_tests.rs real, alpha = 1"),
    dict(fn="dotu", kind="s", n=1024, incx=1, incy=1, x=(0.05, 0.03), y=(-0.3, 0.002),
         src="dot_tests.rs real, n = 1024"),
    dict(fn="dotu", kind="s", n=777, incx=3, incy=2, x=(0.2, -0.001), xalt=True, y=(-0.3, 0.002),
         src="dot_tests.rs real, n = 777 alternating"),
    dict(fn="dotu", kind="s", n=1, incx=5, incy=7, x=(3.14159, 0.0), y=(-2.71828, 0.0),
         src="dot_tests.rs real, n = 1"),
    dict(fn="nrm2", kind="s", n=1024, incx=1, x=(0.05, 0.03), src="nrm2_tests.rs real, n = 1024"),
    dict(fn="nrm2", kind="s", n=777, incx=3, x=(0.2, -0.001), xalt=True, src="nrm2_tests.rs real, n = 777"),
    dict(fn="nrm2", kind="s", n=1, incx=5, x=(-3.14159, 0.0), src="nrm2_tests.rs real, n = 1"),
]

# rot_tests.rs:455-715: (a, b) of the srotg (first four) and drotg (last four)
# cases; both precisions run all eight here
ROTG_CASES = [(3.5, -2.25), (0.0, 5.0), (-4.0, 0.0), (-1.25, -7.5), (12.0, -0.75), (0.0, 3.0), (-5.0, 0.0),
              (-2.0, 9.0)]
# rot_tests.rs:936-999 (srotmg) and 1227-1290 (drotmg): (kind, d1, d2, x1, y1)
ROTMG_CASES = [("s", 1.5, 2.0, 0.75, -1.25), ("s", 1e-3, 3e2, -4.5, 7.25), ("d", 5.0, 0.75, -2.0, 3.0),
               ("d", 1e4, 1e-5, 8.0, -6.0)]


def l1_vectors(case):
    """(x, y) of a L1_CASES entry (y None when the routine has one vector)."""
    x = ramp(case["kind"], case["n"], case["incx"], case["x"], case.get("xalt", False), case.get("plant"))
    y = ramp(case["kind"], case["n"], case["incy"], case["y"]) if "y" in case else None
    return x, y


def rot_cs(case):
    """(c, s) of a rot case: cos / sin of theta in the element precision."""
    real = np.float32 if case["kind"] in "sc" else np.float64
    t = real(case["theta"])
    return real(np.cos(t)), real(np.sin(t))


# ---- symmetric / Hermitian matrix-vector -------------------------------------
# ssymv_tests.rs / dsymv_tests.rs and chemv_tests.rs / zhemv_tests.rs use the
# same closed forms in their element precision; `kind` picks it.
def _real(kind):
    return np.float32 if kind in "sc" else np.float64


def _sym_fill(n, lda, f, stored=None, kind="s"):
    """Column-major n x n buffer: f(R, lo, hi) on the stored triangle,
    mirrored (or NaN in the other triangle when `stored` is 'U' or 'L')."""
    R = _real(kind)
    a = np.zeros(lda * n, R)
    for j in range(n):
        i = np.arange(n)
        lo = np.minimum(i, j).astype(R)
        hi = np.maximum(i, j).astype(R)
        col = np.asarray(f(R, lo, hi), R)
        if stored == "U":
            col = np.where(i <= j, col, R(np.nan))
        elif stored == "L":
            col = np.where(i >= j, col, R(np.nan))
        a[j * lda:j * lda + n] = col
    return a


def symv_matrix(n, lda, kind="s"):
    """ssymv_tests.rs:44-60 / dsymv_tests.rs:46-62 make_symmetric_col_major."""
    return _sym_fill(n, lda, lambda R, lo, hi: R(0.1) + R(0.5) * lo + R(0.25) * hi, kind=kind)


SYMV_COEFFS = [(1.0, 0.0), (0.0, 0.7), (0.75, -0.25), (-0.6, 0.4), (1.1, 0.0), (0.85, 0.1)]  # ssymv_tests.rs:209-216
# (n, lda, [(incx, incy)]): ssymv_tests.rs:227-245, dsymv_tests.rs:230-248
SYMV_SHAPES = [(6, 6, [(1, 1)]), (768, 768, [(1, 1)]), (300, 305, [(1, 1)]),
               (640, 640, [(2, 3), (3, 2), (2, 1)])]


def rvec(kind, length, inc, g):
    """make_strided_vec with |k| g(R, k) in the element precision."""
    R = _real(kind)
    v = np.zeros((length - 1) * inc + 1 if length else 1, R)
    k = np.arange(length).astype(R)
    v[np.arange(length) * inc] = np.asarray(g(R, k), R)
    return v


def symv_x(kind, n, inc):
    return rvec(kind, n, inc, lambda R, k: R(0.2) + R(0.1) * k)


def symv_y(kind, n, inc):
    return rvec(kind, n, inc, lambda R, k: R(-0.3) + R(0.05) * k)


def symv_garbage_cases(kind="s"):
    """ssymv_tests.rs:287-378 / dsymv_tests.rs:294-378: one triangle stored,
    NaN in the other.  (uplo, n, lda, alpha, beta, a, x, y)."""
    up = _sym_fill(200, 203, lambda R, lo, hi: R(0.2) + R(0.3) * lo + R(0.15) * hi, "U", kind)
    lw = _sym_fill(180, 180, lambda R, lo, hi: R(0.17) + R(0.45) * lo + R(0.08) * hi, "L", kind)
    return [
        (0, 200, 203, 0.7, 0.25, up, rvec(kind, 200, 1, lambda R, k: R(0.03) * k - R(0.5)),
         rvec(kind, 200, 1, lambda R, k: R(-0.1) + R(0.002) * k)),
        (1, 180, 180, -0.9, 0.6, lw, rvec(kind, 180, 1, lambda R, k: R(0.2) - R(0.001) * k),
         rvec(kind, 180, 1, lambda R, k: R(0.15) + R(0.004) * k)),
    ]


def cvec(kind, length, inc, gre, gim):
    """make_strided_cvec: element k is (gre(R, k), gim(R, k))."""
    R = _real(kind)
    v = np.zeros((length - 1) * inc + 1 if length else 1, _DT[kind])
    k = np.arange(length).astype(R)
    val = np.empty(length, _DT[kind])
    val.real, val.imag = np.asarray(gre(R, k), R), np.asarray(gim(R, k), R)
    v[np.arange(length) * inc] = val
    return v


def cstrided(length: int, inc: int, fre, fim) -> np.ndarray:
    """chemv_tests.rs:135-152 make_strided_cvec, as complex64."""
    return cvec("c", length, inc, lambda R, k: fre(k), lambda R, k: fim(k))


def _herm(n, lda, fre, fim, stored=None, kind="c"):
    """Column-major complex n x n buffer with re = fre(R, lo, hi) and
    im = fim(R, lo, hi) (0 on the diagonal).  stored None: full Hermitian
    matrix, (re, im) on and above the diagonal and (re, -im) below
    (chemv_tests.rs:47-73); 'U' / 'L': only that triangle holds (re, im),
    the other NaN (chemv_tests.rs:76-133)."""
    R = _real(kind)
    a = np.zeros(lda * n, _DT[kind])
    for j in range(n):
        i = np.arange(n)
        lo = np.minimum(i, j).astype(R)
        hi = np.maximum(i, j).astype(R)
        re = np.asarray(fre(R, lo, hi), R)
        im = np.where(i == j, R(0.0), np.asarray(fim(R, lo, hi), R)).astype(R)
        if stored is None:
            im = np.where(i <= j, im, -im)
        val = np.empty(n, _DT[kind])
        val.real, val.imag = re, im
        if stored == "U":
            val[i > j] = complex(np.nan, np.nan)
        elif stored == "L":
            val[i < j] = complex(np.nan, np.nan)
        a[j * lda:j * lda + n] = val
    return a


def hemv_matrix(n, lda, kind="c"):
    """chemv_tests.rs:47-73 / zhemv_tests.rs:48-74 make_hermitian_col_major:
    upper (i <= j) holds (re, im), lower holds (re, -im)."""
    return _herm(n, lda, lambda R, lo, hi: R(0.10) + R(0.25) * lo + R(0.15) * hi,
                 lambda R, lo, hi: R(0.04) + R(0.02) * (hi - lo), kind=kind)


# chemv_tests.rs:262-269 as (alpha, beta)
HEMV_COEFFS = [(1.0 + 0j, 0j), (0j, 0.7 - 0.1j), (0.75 - 0.10j, -0.25 + 0.15j), (-0.6 + 0.2j, 0.4 - 0.1j),
               (1.25 + 0j, -0.5 + 0j), (0.85 - 0.1j, 0.1 + 0.05j)]
# zhemv_tests.rs:260-268
ZHEMV_COEFFS = [(1.0 + 0j, 0j), (0j, -0.75 + 0.2j), (0.75 - 0.10j, -0.25 + 0.15j), (-0.6 + 0.2j, 0.4 - 0.1j),
                (1.25 + 0j, -0.5 + 0j), (0.85 - 0.1j, 0.1 + 0.05j), (1.1 - 0.2j, 0j)]
# (n, lda, [(incx, incy)]): chemv_tests.rs:281-299, zhemv_tests.rs:280-298
HEMV_SHAPES = [(6, 6, [(1, 1)]), (640, 640, [(1, 1)]), (300, 305, [(1, 1)]),
               (384, 384, [(2, 3), (3, 2), (2, 1)])]


def hemv_x(length, inc, kind="c"):
    return cvec(kind, length, inc, lambda R, k: R(0.2) + R(0.1) * k, lambda R, k: R(-0.3) + R(0.05) * k)


def hemv_y(length, inc, kind="c"):
    return cvec(kind, length, inc, lambda R, k: R(-0.3) + R(0.05) * k, lambda R, k: R(0.1) - R(0.02) * k)


def hemv_garbage_cases(kind="c"):
    """chemv_tests.rs:360-478 / zhemv_tests.rs:361-478: one triangle stored,
    NaN in the other.  (uplo, n, lda, alpha, beta, a, x, y)."""
    up = _herm(200, 203, lambda R, lo, hi: R(0.20) + R(0.30) * lo + R(0.15) * hi,
               lambda R, lo, hi: R(0.05) + R(0.01) * (hi - lo), "U", kind)
    lw = _herm(180, 180, lambda R, lo, hi: R(0.17) + R(0.45) * lo + R(0.08) * hi,
               lambda R, lo, hi: R(-0.03) - R(0.02) * (hi - lo), "L", kind)
    return [
        (0, 200, 203, 0.7 + 0.1j, 0.25 - 0.05j, up,
         cvec(kind, 200, 1, lambda R, k: R(0.03) * k - R(0.5), lambda R, k: R(0.02) - R(0.01) * k),
         cvec(kind, 200, 1, lambda R, k: R(-0.1) + R(0.002) * k, lambda R, k: R(0.05) - R(0.003) * k)),
        (1, 180, 180, -0.9 + 0.2j, 0.6 - 0.1j, lw,
         cvec(kind, 180, 1, lambda R, k: R(0.2) - R(0.001) * k, lambda R, k: R(-0.03) + R(0.004) * k),
         cvec(kind, 180, 1, lambda R, k: R(0.15) + R(0.004) * k, lambda R, k: R(-0.02) + R(0.003) * k)),
    ]


# ---- strmv_tests.rs:61-160, 200-240 ------------------------------------------
def trmv_matrix(n, lda, uplo, diag):
    """build_matrix: make_upper / make_lower, with a deliberately wrong
    diagonal when diag is unit (CORAL diag 0) so that it must be ignored."""
    a = np.zeros(lda * n, np.float32)
    for j in range(n):
        i = np.arange(n).astype(np.float32)
        if uplo == 0:
            col = f32(0.2) + i * f32(0.3) + f32(j) * f32(0.15)
            rows = np.arange(n) <= j
        else:
            col = f32(-0.1) + i * f32(0.25) - f32(j) * f32(0.2)
            rows = np.arange(n) >= j
        a[j * lda:j * lda + n] = np.where(rows, col, f32(0.0))
    if diag == 0:
        for i in range(n):
            a[i + i * lda] = (f32(7.5) + f32(i) * f32(0.1)) if uplo == 0 else (f32(-9.0) + f32(i) * f32(0.05))
    return a


def trmv_x(n, inc):
    return strided(n, inc, lambda k: f32(0.1) + f32(0.2) * k)


# (n, lda, incs): strmv_tests.rs:226-240 (trans N, T and C; C is T for real data)
TRMV_SHAPES = [(7, 7, [1]), (1024, 1024, [1]), (640, 640, [2, 3])]


# ---- sger_tests.rs, ssyr_tests.rs, ssyr2_tests.rs ------------------------------
def ger_matrix(m, n, lda):
    """sger_tests.rs:33-48 make_matrix (the same ramp as sgemv's)."""
    return colmajor(m, n, lda, lambda i, j: f32(0.1) + i * f32(0.5) + j * f32(0.25))


# (m, n, lda, incx, incy, alpha, x ramp, y ramp): sger_tests.rs:128-231
GER_CASES = [
    (7, 5, 7, 1, 1, 1.25, (0.2, 0.1), (-0.1, 0.07)),
    (1024, 768, 1024, 1, 1, -0.37, (0.05, 0.002), (0.4, -0.003)),
    (512, 1024, 512, 1, 1, 0.93, (-0.2, 0.0015), (0.1, 0.0020)),
    (9, 4, 12, 2, 3, -0.85, (0.05, 0.03), (0.4, -0.02)),
    (300, 200, 305, 1, 1, 0.0, (0.11, 0.01), (0.07, -0.01)),
]


def syr_matrix(n, lda, kind="s"):
    """ssyr_tests.rs:55-70 / ssyr2_tests.rs:57-72 make_symmetric_col_major."""
    return _sym_fill(n, lda, lambda R, lo, hi: R(0.1) + R(0.5) * lo + R(0.25) * hi, kind=kind)


# (uplo, n, lda, incx, alpha, x ramp): ssyr_tests.rs:178-244
SYR_CASES = [
    (0, 7, 7, 1, 1.25, (0.2, 0.1)),
    (1, 7, 7, 1, -0.8, (-0.3, 0.05)),
    (0, 1024, 1024, 1, -0.37, (0.05, 0.002)),
    (1, 512, 512, 1, 0.93, (-0.2, 0.0015)),
    (1, 9, 12, 2, -0.85, (0.05, 0.03)),
    (0, 300, 305, 1, 0.0, (0.11, 0.01)),
]

# (uplo, n, lda, incx, incy, alpha, x ramp, y ramp): ssyr2_tests.rs:178-245, 350-361
SYR2_CASES = [
    (0, 7, 7, 1, 1, 1.25, (0.2, 0.1), (-0.3, 0.05)),
    (1, 7, 7, 1, 1, -0.8, (-0.2, 0.07), (0.4, -0.055)),
    (0, 1024, 1024, 1, 1, -0.37, (0.05, 0.002), (0.4, -0.003)),
    (1, 512, 512, 1, 1, 0.93, (-0.2, 0.0015), (0.1, 0.0020)),
    (1, 9, 12, 2, 3, -0.85, (0.05, 0.03), (0.4, -0.02)),
    (0, 300, 305, 1, 1, 0.0, (0.11, 0.01), (0.07, -0.01)),
]


def ramp32(n, inc, g):
    """make_strided_vec with |k| g0 + g1 * k in f32."""
    return strided(n, inc, lambda k: f32(g[0]) + f32(g[1]) * k)


def sample_positions(rows, cols, count=4096, seed=0):
    """Fixed (row, col) positions at which large rank-update results are
    stored: every entry when the matrix has at most `count`, else a seeded
    sample."""
    if rows * cols <= count:
        r, c = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
        return r.ravel(), c.ravel()
    rng = np.random.default_rng(seed + rows * 7919 + cols)
    return rng.integers(0, rows, count), rng.integers(0, cols, count)


# ---- d/c/z matrix-vector: dgemv/cgemv/zgemv_tests.rs -------------------------
def cm_k(kind, rows, cols, ld, fre, fim=None):
    """Column-major buffer in the element precision: element (i, j) is
    fre(R, i, j) (+ 1j * fim(R, i, j) for complex kinds)."""
    R = _real(kind)
    a = np.zeros(ld * cols, _DT[kind])
    i = np.arange(rows).astype(R)
    for j in range(cols):
        jj = R(j)
        if kind in "sd":
            a[j * ld:j * ld + rows] = fre(R, i, jj)
        else:
            col = np.empty(rows, _DT[kind])
            col.real, col.imag = fre(R, i, jj), fim(R, i, jj)
            a[j * ld:j * ld + rows] = col
    return a


def gemv_matrix_k(kind, m, n, lda):
    """dgemv_tests.rs:50-62; cgemv_tests.rs:48-63 / zgemv_tests.rs:51-66 add
    im = -0.2 + 0.3 i - 0.15 j."""
    return cm_k(kind, m, n, lda, lambda R, i, j: R(0.1) + i * R(0.5) + j * R(0.25),
                lambda R, i, j: R(-0.2) + i * R(0.3) - j * R(0.15))


def gemv_x_k(kind, length, inc):
    if kind in "sd":
        return rvec(kind, length, inc, lambda R, k: R(0.2) + R(0.1) * k)
    return cvec(kind, length, inc, lambda R, k: R(0.2) + R(0.1) * k, lambda R, k: R(-0.05) * k)


def gemv_y_k(kind, length, inc):
    if kind in "sd":
        return rvec(kind, length, inc, lambda R, k: R(-0.3) + R(0.05) * k)
    return cvec(kind, length, inc, lambda R, k: R(-0.3) + R(0.05) * k, lambda R, k: R(0.02) * k)


# per kind: (ops, coefficients, shapes (m, n, lda, [(incx, incy)]), rtol, atol)
GEMV_DCZ = {
    "d": ((0, 1), [(1.0, 0.0), (0.0, -0.75), (0.75, -0.25), (-0.6, 0.4), (1.1, 0.0), (0.85, 0.1)],
          [(5, 4, 5, [(1, 1)]), (1024, 512, 1024, [(1, 1), (2, 3), (3, 2), (2, 1)]), (256, 1024, 263, [(1, 1)]),
           (640, 320, 640, [(1, 1)])], 1e-13, 1e-13),                      # dgemv_tests.rs:117-118, 193-246
    "c": ((0, 1, 2), [(1.0 + 0j, 0j), (0j, 0.7 - 0.1j), (0.75 - 0.25j, 0.5 + 0j), (-0.5 + 0.2j, 0.3 - 0.15j),
                      (1.1 - 0.6j, 0j), (0.3 + 0.7j, 0.1 - 0.2j)],
          [(5, 4, 5, [(1, 1)]), (384, 256, 384, [(1, 1)]), (256, 512, 263, [(1, 1)]),
           (300, 200, 305, [(2, 1), (1, 3), (2, 3)]), (64, 192, 64, [(1, 1)])], 5e-3, 1e-6),  # cgemv_tests.rs:125-126, 192-255
    "z": ((0, 1, 2), [(1.0 + 0j, 0j), (0j, -0.75 + 0.2j), (0.75 - 0.10j, -0.25 + 0.05j), (-0.6 + 0.2j, 0.4 - 0.1j),
                      (1.1 - 0.6j, 0j), (0.85 - 0.2j, 0.1 + 0j)],
          [(5, 4, 5, [(1, 1)]), (384, 256, 384, [(1, 1)]), (256, 512, 263, [(1, 1)]),
           (512, 256, 512, [(2, 3), (3, 2), (2, 1)]), (640, 320, 640, [(1, 1)])], 1e-11, 1e-12),  # zgemv_tests.rs:138-139, 218-273
}


# ---- d/c/z triangular multiply and solve -------------------------------------
def tri_fill(kind, n, lda, uplo, fdiag, foff):
    """Triangle `uplo` (0 upper, 1 lower) of a column-major buffer:
    fdiag(R, i) on the diagonal, foff(R, d) off it, d = |i - j| as R.
    Each callable returns a real value or a (re, im) pair."""
    R = _real(kind)
    a = np.zeros(lda * n, _DT[kind])
    for j in range(n):
        rows = np.arange(0, j + 1) if uplo == 0 else np.arange(j, n)
        d = np.abs(rows - j).astype(R)
        ii = rows.astype(R)
        off, dia = foff(R, d), fdiag(R, ii)
        if kind in "sd":
            col = np.where(rows == j, dia, off)
        else:
            col = np.empty(rows.size, _DT[kind])
            col.real = np.where(rows == j, dia[0], off[0])
            col.imag = np.where(rows == j, dia[1], off[1])
        a[j * lda + rows] = col
    return a


def set_diag(kind, a, n, lda, f):
    R = _real(kind)
    for i in range(n):
        v = f(R, R(i))
        a[i + i * lda] = v if kind in "sd" else complex(v[0], v[1])
    return a


def trmv_matrix_k(kind, n, lda, uplo, diag):
    """dtrmv_tests.rs:63-176 (the strmv closed forms in f64);
    ctrmv_tests.rs / ztrmv_tests.rs:63-155, 215-242 build_matrix."""
    if kind in "sd":
        R = _real(kind)
        f = (lambda i, j: R(0.2) + i * R(0.3) + j * R(0.15)) if uplo == 0 else \
            (lambda i, j: R(-0.1) + i * R(0.25) - j * R(0.2))
        a = cm_k(kind, n, n, lda, lambda R_, i, j: f(i, j))
        r, c = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        keep = (r <= c) if uplo == 0 else (r >= c)
        a[(r + c * lda)[~keep]] = 0.0
        if diag == 0:
            set_diag(kind, a, n, lda, (lambda R_, i: R_(7.5) + i * R_(0.1)) if uplo == 0 else
                     (lambda R_, i: R_(-9.0) + i * R_(0.05)))
        return a
    return _ctri(kind, n, lda, uplo, diag, trsv=False)


def _ctri(kind, n, lda, uplo, diag, trsv):
    """The complex triangles of ctrmv/ztrmv_tests.rs:63-155 and
    ctrsv/ztrsv_tests.rs:91-183 (identical forms), with build_matrix's
    planted diagonal for unit calls (its lower imaginary part is 2.1 - 0.03 i
    in the multiply tests, 4.2 - 0.03 i in the solve tests)."""
    if diag == 1:
        if uplo == 0:
            a = tri_fill(kind, n, lda, 0, lambda R, i: (R(1.0) + R(0.02) * i, R(0.01) - R(0.005) * i),
                         lambda R, d: (R(0.01) / (R(1.0) + d), R(-0.008) / (R(1.0) + d)))
        else:
            a = tri_fill(kind, n, lda, 1, lambda R, i: (R(1.0) + R(0.02) * i, R(-0.012) + R(0.004) * i),
                         lambda R, d: (R(0.01) / (R(1.0) + d), R(0.007) / (R(1.0) + d)))
        return a
    if uplo == 0:
        a = tri_fill(kind, n, lda, 0, lambda R, i: (R(2.5) + R(0.05) * i, R(-1.7) + R(0.01) * i),
                     lambda R, d: (R(5e-4) * (R(1.0) + d), R(-3e-4) * (R(1.0) + d)))
        return set_diag(kind, a, n, lda, lambda R, i: (R(7.5) + i * R(0.1), R(-3.2) + i * R(0.07)))
    a = tri_fill(kind, n, lda, 1, lambda R, i: (R(-2.0) + R(0.04) * i, R(1.2) - R(0.02) * i),
                 lambda R, d: (R(6e-4) * (R(1.0) + d), R(4e-4) * (R(1.0) + d)))
    return set_diag(kind, a, n, lda, lambda R, i: (R(-9.0) + i * R(0.05),
                                                     (R(4.2) if trsv else R(2.1)) - i * R(0.03)))


def trmv_x_k(kind, n, inc):
    if kind in "sd":
        return rvec(kind, n, inc, lambda R, k: R(0.1) + R(0.2) * k)
    return cvec(kind, n, inc, lambda R, k: R(0.1) + R(0.2) * k, lambda R, k: R(-0.05) + R(0.03) * k)


# per kind: (ops, shapes (n, lda, incs), rtol, atol)
TRMV_DCZ = {
    "d": ((0, 1, 2), [(7, 7, [1]), (1024, 1024, [1]), (640, 640, [2, 3])], 1e-13, 1e-13),   # dtrmv_tests.rs:154-155, 220-258
    "c": ((0, 1, 2), [(7, 7, [1]), (768, 768, [1]), (256, 261, [1]), (384, 384, [2, 3, 4])], 1e-5, 1e-5),  # ctrmv_tests.rs:213-214, 295-337
    "z": ((0, 1, 2), [(7, 7, [1]), (768, 768, [1]), (256, 261, [1]), (384, 384, [2, 3, 4])], 1e-13, 1e-13),  # ztrmv_tests.rs:213-214, 295-337
}


def trsv_matrix_k(kind, n, lda, uplo, diag):
    """strsv_tests.rs / dtrsv_tests.rs:64-166, 216-241 build_matrix (unit
    calls get make_upper_unit / make_lower_unit with a planted diagonal);
    c/z: ctrsv/ztrsv_tests.rs 91-183, 244-272."""
    if kind in "cz":
        return _ctri(kind, n, lda, uplo, diag, trsv=True)
    if diag == 1:
        return tri_fill(kind, n, lda, uplo, lambda R, i: R(1.0) + R(0.02) * i, lambda R, d: R(0.01) / (R(1.0) + d))
    if uplo == 0:
        a = tri_fill(kind, n, lda, 0, lambda R, i: R(1.0) + R(0.05) * i, lambda R, d: R(5e-4) * (R(1.0) + d))
        return set_diag(kind, a, n, lda, lambda R, i: R(7.5) + i * R(0.1))
    a = tri_fill(kind, n, lda, 1, lambda R, i: R(1.0) - R(0.03) * i, lambda R, d: R(6e-4) * (R(1.0) + d))
    return set_diag(kind, a, n, lda, lambda R, i: R(-9.0) + i * R(0.05))


def trsv_x_k(kind, n, inc):
    if kind in "sd":
        return rvec(kind, n, inc, lambda R, k: R(0.05) + R(0.01) * k)
    return cvec(kind, n, inc, lambda R, k: R(0.1) + R(0.2) * k, lambda R, k: R(-0.05) + R(0.03) * k)


TRSV_DCZ = {
    "d": ((0, 1), [(7, 7, [1]), (1024, 1024, [1]), (640, 640, [2, 3, 4]), (127, 132, [1])], 1e-12, 1e-12),  # dtrsv_tests.rs:213-214, 285-332
    "c": ((0, 1, 2), [(7, 7, [1]), (760, 768, [1]), (384, 384, [2, 3, 4]), (256, 263, [1])], 1e-2, 1e-3),  # ctrsv_tests.rs:241-242, 320-363
    "z": ((0, 1, 2), [(7, 7, [1]), (768, 768, [1]), (384, 384, [2, 3, 4]), (256, 263, [1])], 1e-11, 1e-11),  # ztrsv_tests.rs:241-242, 320-363
}


def sample_index(length, count=96):
    """Fixed positions of a result vector stored in the golden file: all of
    it up to `count` entries, else the first and last 8 and an even spread
    between them."""
    if length <= count:
        return np.arange(length)
    mid = np.linspace(8, length - 9, count - 16).astype(np.int64)
    return np.unique(np.concatenate([np.arange(8), mid, np.arange(length - 8, length)]))


# ---- d/c/z rank updates: dger, dsyr, dsyr2, {c,z}ger{u,c}, {c,z}her, {c,z}her2 ----
# dger/dsyr/dsyr2_tests.rs run the sger/ssyr/ssyr2 case tables in f64
# (GER_CASES, SYR_CASES, SYR2_CASES); tolerances (rtol, atol):
RANK_TOL = {"sger": (1e-6, 1e-6), "dger": (1e-13, 1e-13),        # sger/dger_tests.rs:82-83, 81-82
            "ssyr": (1e-6, 1e-5), "dsyr": (1e-6, 1e-5),          # ssyr/dsyr_tests.rs:129-130, 128-129
            "ssyr2": (1e-6, 1e-5), "dsyr2": (1e-6, 1e-5),        # ssyr2/dsyr2_tests.rs:131-132
            "cger": (1e-6, 1e-6), "zger": (1e-12, 1e-12),        # cger/zger_tests.rs:118-119, 111-112
            "cher": (1e-5, 1e-6), "zher": (1e-13, 1e-13),        # cher/zher_tests.rs:147-148, 149-150
            "cher2": (1e-5, 1e-6), "zher2": (1e-13, 1e-13)}      # cher2/zher2_tests.rs:148-149, 156-157


def rank_vec(kind, n, inc, g):
    """Ramp g = (a, b) for real kinds, (re0, re1, im0, im1) for complex."""
    if kind in "sd":
        return rvec(kind, n, inc, lambda R, k: R(g[0]) + R(g[1]) * k)
    return cvec(kind, n, inc, lambda R, k: R(g[0]) + R(g[1]) * k, lambda R, k: R(g[2]) + R(g[3]) * k)


# (m, n, lda, incx, incy, alpha geru, alpha gerc, x ramp, y ramp):
# cger_tests.rs / zger_tests.rs run_contiguous_sets, run_strided_padded,
# run_alpha_zero(300, 200, 305)
CGER_CASES = [
    (7, 5, 7, 1, 1, 1.25 - 0.40j, 0.85 + 0.35j, (0.20, 0.10, -0.30, 0.05), (-0.10, 0.07, 0.20, -0.04)),
    (1024, 768, 1024, 1, 1, -0.37 + 0.21j, -0.21 + 0.44j, (0.05, 0.002, -0.02, 0.001), (0.40, -0.003, 0.10, 0.002)),
    (512, 1024, 512, 1, 1, 0.93 - 0.61j, 0.37 - 0.72j, (-0.20, 0.0015, 0.30, -0.0007), (0.10, 0.0020, 0.20, 0.0010)),
    (9, 4, 12, 2, 3, -0.85 + 0j, 0.65 + 0.10j, (0.05, 0.03, 0.04, -0.01), (0.40, -0.02, -0.30, 0.05)),
    (300, 200, 305, 1, 1, 0j, 0j, (0.11, 0.01, -0.02, 0.003), (0.07, -0.01, 0.05, 0.004)),
]

# (uplo, n, lda, incx, alpha, x ramp): cher_tests.rs / zher_tests.rs
# run_small_and_large, run_lower_padded_strided, the alpha = 0 case
HER_CASES = [
    (0, 6, 6, 1, 0.9, (0.2, 0.1, -0.05, 0.02)),
    (0, 512, 512, 1, -0.37, (0.03, 0.001, -0.02, 0.0007)),
    (1, 7, 7, 1, -0.8, (-0.1, 0.03, 0.07, -0.01)),
    (1, 256, 256, 1, 0.93, (-0.02, 0.0005, 0.01, -0.0003)),
    (1, 9, 12, 2, -0.85, (0.05, 0.03, -0.02, 0.01)),
    (0, 64, 69, 1, 0.0, (0.11, 0.01, -0.07, 0.004)),
]

# (uplo, n, lda, incx, incy, alpha, x ramp, y ramp): cher2_tests.rs /
# zher2_tests.rs run_small_and_large, run_lower_padded_strided,
# run_alpha_zero_does_nothing
HER2_CASES = [
    (0, 7, 7, 1, 1, 1.10 - 0.35j, (0.2, 0.10, -0.05, 0.02), (-0.3, 0.05, 0.07, -0.01)),
    (0, 1024, 1024, 1, 1, -0.37 + 0.20j, (0.05, 0.002, -0.02, 0.0007), (0.40, -0.003, 0.01, -0.0005)),
    (1, 7, 7, 1, 1, -0.80 + 0.50j, (-0.2, 0.07, 0.06, -0.01), (0.4, -0.055, -0.03, 0.02)),
    (1, 512, 512, 1, 1, 0.93 - 0.10j, (-0.20, 0.0015, 0.03, -0.0004), (0.10, 0.0020, -0.01, 0.0003)),
    (1, 9, 12, 2, 3, -0.85 + 0.25j, (0.05, 0.03, -0.02, 0.01), (0.40, -0.02, 0.03, -0.01)),
    (0, 300, 305, 1, 1, 0j, (0.11, 0.01, -0.07, 0.004), (0.08, -0.01, 0.02, 0.003)),
]


# ---- d/c/z GEMM: dgemm_tests.rs, cgemm_tests.rs, zgemm_tests.rs ------------------
def gemm_operands_k(kind, op_a, op_b, m, n, k, lda, ldb, ldc):
    """dgemm_tests.rs:112-114 (the sgemm closed forms in f64);
    cgemm_tests.rs:136-152 / zgemm_tests.rs:133-149 add the imaginary ramps."""
    a_rows, a_cols = (m, k) if op_a == 0 else (k, m)
    b_rows, b_cols = (k, n) if op_b == 0 else (n, k)
    a = cm_k(kind, a_rows, a_cols, lda, lambda R, i, j: R(0.1) + i * R(0.25) + j * R(0.125),
             lambda R, i, j: R(-0.05) + i * R(0.20) - j * R(0.075))
    b = cm_k(kind, b_rows, b_cols, ldb, lambda R, i, j: R(-0.2) + i * R(0.05) - j * R(0.075),
             lambda R, i, j: R(0.15) - i * R(0.03) + j * R(0.02))
    c = cm_k(kind, m, n, ldc, lambda R, i, j: R(0.3) - i * R(0.01) + j * R(0.02),
             lambda R, i, j: R(-0.1) + i * R(0.015) - j * R(0.025))
    return a, b, c


# dgemm_tests.rs:143-186: the four real op pairs for each (alpha, beta), and
# (C, N) with the first pair and (N, C) with the second.
DGEMM_CASES = [((oa, ob), ci) for ci in range(4) for (oa, ob) in [(0, 0), (0, 1), (1, 0), (1, 1)]] + \
    [((2, 0), 0), ((0, 2), 1)]
DGEMM_COEFFS = GEMM_ALPHA_BETA
# cgemm_tests.rs:188-223 / zgemm_tests.rs:184-219: nine op pairs x four
# (alpha, beta)
CGEMM_OPS = [(0, 0), (0, 1), (1, 0), (1, 1), (0, 2), (1, 2), (2, 0), (2, 1), (2, 2)]
CGEMM_COEFFS = [(1.0 + 0j, 0j), (0.5 + 0.25j, 1.0 + 0j), (0.75 - 0.25j, -0.5 + 0.3j), (0j, 0.7 - 0.2j)]
GEMM_TOL = {"d": (1e-12, 1e-12), "c": (3e-3, 2e-3), "z": (3e-11, 2e-11)}  # dgemm:83-84, cgemm:109-110, zgemm:106-107


def gemm_cases_k(kind):
    """((op_a, op_b), (alpha, beta)) pairs of one kind's test file."""
    if kind == "d":
        return [(ops, DGEMM_COEFFS[ci]) for ops, ci in DGEMM_CASES]
    return [(ops, ab) for ab in CGEMM_COEFFS for ops in CGEMM_OPS]


# ---- rank updates applied twice (each file's run_accumulate_twice) -------------
# real: (m or n, alpha1, alpha2, x1, y1, x2, y2) with ramps (a, b); the ger
# form is 64 x 48, the syr/syr2 forms 64 x 64 upper (sger/ssyr/ssyr2 and
# dger/dsyr/dsyr2_tests.rs)
ACC_REAL = dict(m=64, n=48, alpha=(1.2, -0.7), x1=(0.2, 0.01), y1=(-0.1, 0.02), x2=(-0.3, 0.03), y2=(0.4, -0.01))
# cger/zger_tests.rs run_accumulate_twice: alphas per form (geru, gerc)
ACC_CGER = dict(m=64, n=48, alpha={0: (1.20 - 0.30j, -0.70 + 0.15j), 1: (0.60 + 0.40j, -0.70 + 0.20j)},
                x1=(0.20, 0.01, -0.10, 0.02), y1=(-0.10, 0.02, 0.40, -0.01),
                x2=(-0.30, 0.03, 0.25, -0.02), y2=(0.40, -0.01, -0.20, 0.03))
# cher/zher_tests.rs (n = 33, upper) and cher2/zher2_tests.rs (n = 64, upper)
ACC_HER = dict(n=33, alpha=(1.2, -0.7), x1=(0.20, 0.01, -0.03, 0.005), x2=(-0.30, 0.03, 0.06, -0.004))
ACC_HER2 = dict(n=64, alpha=(1.20 + 0.30j, -0.70 - 0.20j), x1=(0.20, 0.01, -0.03, 0.005),
                y1=(-0.10, 0.02, 0.04, -0.003), x2=(-0.30, 0.03, 0.06, -0.004), y2=(0.40, -0.01, -0.02, 0.002))


# ---- the triangular files' single-case tests -------------------------------------
def padded_k(kind, n, lda, trsv):
    """Both triangles populated: strsv/dtrsv make_padded (diagonal
    1 + 0.02 i, 0.01 / (1 + d) off it), ctrsv/ztrsv make_padded_c32, and for
    the multiply tests strmv/dtrmv make_padded_col_major (lower
    0.1 + 0.2 i + 0.1 j, upper 0.1 + 0.1 i + 0.2 j)."""
    R = _real(kind)
    if not trsv:
        return cm_k(kind, n, n, lda, lambda R_, i, j: np.where(i >= j, R_(0.1) + i * R_(0.2) + j * R_(0.1),
                                                                R_(0.1) + i * R_(0.1) + j * R_(0.2)))
    a = np.zeros(lda * n, _DT[kind])
    for j in range(n):
        i = np.arange(n)
        d = np.abs(i - j).astype(R)
        ii = i.astype(R)
        re = np.where(i == j, R(1.0) + R(0.02) * ii, R(0.01) / (R(1.0) + d))
        if kind in "sd":
            a[j * lda:j * lda + n] = re
            continue
        im = np.where(i == j, R(0.01) - R(0.005) * ii,
                      np.where(i < j, R(-0.008) / (R(1.0) + d), R(0.007) / (R(1.0) + d)))
        col = np.empty(n, _DT[kind])
        col.real, col.imag = re, im
        a[j * lda:j * lda + n] = col
    return a


def tri_special_cases(kind, trsv):
    """(name, uplo, trans, diag, n, lda, a, x) of lower_transpose_padded /
    padded_lower_transpose, and for strsv/dtrsv unitdiag_upper_notranspose
    and unitdiag_lower_transpose."""
    if kind in "sd":
        lda = 132
        x = rvec(kind, 127, 1, lambda R, k: R(0.3) - R(0.006) * k)
    else:
        lda = 134
        x = cvec(kind, 127, 1, lambda R, k: R(0.3) - R(0.006) * k, lambda R, k: R(-0.12) + R(0.003) * k)
    out = [("ltp", 1, 1, 1, 127, lda, padded_k(kind, 127, lda, trsv), x)]
    if trsv and kind in "sd":
        out.append(("uun", 0, 0, 0, 40, 40, trsv_matrix_k(kind, 40, 40, 0, 0),
                    rvec(kind, 40, 1, lambda R, k: R(0.2) + R(0.01) * k)))
        out.append(("lut", 1, 1, 0, 48, 48, trsv_matrix_k(kind, 48, 48, 1, 0),
                    rvec(kind, 48, 1, lambda R, k: R(-0.1) + R(0.02) * k)))
    return out


# Edge shapes of the level-1 files (n = 0, and n = 1 with increments past 1),
# for every kind and routine, checked against the oracle only (golden keys
# l1e_c<i>): a one-element vector of 3.14159 (x) and -2.71828 (y).
L1_EDGE_CASES = []
for _k in "sdcz":
    _x = (3.14159, 0.0) if _k in "sd" else (3.14159, 0.0, -0.5, 0.0)
    _y = (-2.71828, 0.0) if _k in "sd" else (-2.71828, 0.0, 0.25, 0.0)
    for _n, _ix, _iy in ((0, 1, 1), (1, 5, 7)):
        _src = f"level-1 edge, n = {_n}"
        L1_EDGE_CASES += [
            dict(fn="axpy", kind=_k, n=_n, incx=_ix, incy=_iy, alpha=1.23 if _k in "sd" else 1.23 - 0.5j, x=_x, y=_y,
                 src=_src),
            dict(fn="scal", kind=_k, n=_n, incx=_ix, alpha=1.23 if _k in "sd" else 1.23 - 0.5j, x=_x, src=_src),
            dict(fn="dotu", kind=_k, n=_n, incx=_ix, incy=_iy, x=_x, y=_y, src=_src),
            dict(fn="asum", kind=_k, n=_n, incx=_ix, x=_x, src=_src),
            dict(fn="nrm2", kind=_k, n=_n, incx=_ix, x=_x, src=_src),
            dict(fn="iamax", kind=_k, n=_n, incx=_ix, x=_x, src=_src),
        ]
        if _k in "cz":
            L1_EDGE_CASES.append(dict(fn="dotc", kind=_k, n=_n, incx=_ix, incy=_iy, x=_x, y=_y, src=_src))
