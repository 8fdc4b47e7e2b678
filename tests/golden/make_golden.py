"""Generates tests/golden/golden.npz: expected outputs of the reference's own
fixture cases computed by CBLAS-class BLAS (scipy's OpenBLAS 0.3.x), the same
class of oracle the reference's tests link (blas-src / openblas-src, see
coral-aarch64/Cargo.toml and tests/level3/sgemm_tests.rs:1-2).

Inputs are the closed-form generators in fixtures.py, rebuilt by the tests;
only outputs are stored.  Run from the repo root:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np
from scipy.linalg import blas

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import fixtures as fx  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")


def logical(buf, rows, cols, ld):
    return np.asfortranarray(buf.reshape(cols, ld).T[:rows, :])


def main() -> None:
    g: dict[str, np.ndarray] = {}
    # ---- SGEMM: small fixture shapes x ops x (alpha, beta), + ConjugateTranspose cases.
    for si, (m, n, k, lda_n, lda_t, ldb_n, ldb_t, ldc) in enumerate(fx.GEMM_SHAPES[:3]):
        for (op_a, op_b) in [(0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (0, 2)]:
            lda = lda_n if op_a == 0 else lda_t
            ldb = ldb_n if op_b == 0 else ldb_t
            a, b, c = fx.gemm_operands(op_a, op_b, m, n, k, lda, ldb, ldc)
            A = logical(a, *((m, k) if op_a == 0 else (k, m)), lda)
            B = logical(b, *((k, n) if op_b == 0 else (n, k)), ldb)
            Cm = logical(c, m, n, ldc)
            for ci, (alpha, beta) in enumerate(fx.GEMM_ALPHA_BETA):
                r = blas.sgemm(alpha, A, B, beta=beta, c=Cm.copy(), trans_a=int(op_a != 0),
                               trans_b=int(op_b != 0))
                g[f"sgemm_s{si}_{op_a}{op_b}_c{ci}"] = np.asarray(r, np.float32).ravel(order="F")
    # ---- SGEMV
    for si, (m, n, lda, strides) in enumerate(fx.GEMV_SHAPES):
        a = fx.gemv_matrix(m, n, lda)
        A = logical(a, m, n, lda)
        for (incx, incy) in strides:
            for trans in (0, 1):
                xl, yl = (n, m) if trans == 0 else (m, n)
                x = fx.gemv_x(xl, incx)
                y0 = fx.gemv_y(yl, incy)
                for ci, (alpha, beta) in enumerate(fx.GEMV_COEFFS):
                    r = blas.sgemv(alpha, A, x, beta=beta, y=y0.copy(), incx=incx, incy=incy,
                                   trans=trans)
                    g[f"sgemv_s{si}_{incx}{incy}_t{trans}_c{ci}"] = np.asarray(r, np.float32)[::incy][:yl]
    # ---- STRSV (uplo 0 upper, 1 lower; CORAL diag 0 = unit, 1 = non-unit)
    for si, (n, lda, incs) in enumerate(fx.TRSV_SHAPES):
        for uplo in (0, 1):
            a = fx.trsv_matrix(n, lda, uplo)
            A = logical(a, n, n, lda)
            for inc in incs:
                x = fx.trsv_x(n, inc)
                for trans in (0, 1):
                    for diag in (0, 1):
                        r = blas.strsv(A, x.copy(), incx=inc, lower=uplo, trans=trans,
                                       diag=1 if diag == 0 else 0)
                        g[f"strsv_s{si}_u{uplo}_i{inc}_t{trans}_d{diag}"] = np.asarray(r, np.float32)[::inc][:n]
    # ---- ISAMAX planted maxima
    for ci, (n, inc, x) in enumerate(fx.isamax_cases()):
        idx = 0 if n == 0 else int(blas.isamax(x, n=n, incx=inc))
        g[f"isamax_c{ci}"] = np.array([idx], np.int64)
    np.savez_compressed(OUT, **g)
    print(f"wrote {len(g)} arrays to {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
