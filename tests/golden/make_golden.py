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


def S(v):
    """The stored positions of a result vector (fixtures.sample_index)."""
    return v[fx.sample_index(v.size)]


def l1_reference(case) -> np.ndarray:
    """OpenBLAS result of one L1_CASES entry: the updated vector(s) or the
    scalar, as a flat array."""
    kind, n, fn = case["kind"], case["n"], case["fn"]
    x, y = fx.l1_vectors(case)
    incx, incy = case["incx"], case.get("incy", 1)
    pre = {"s": "s", "d": "d", "c": "c", "z": "z"}[kind]
    if fn == "axpy":
        return getattr(blas, pre + "axpy")(x, y.copy(), n=n, a=case["alpha"], incx=incx, incy=incy)
    if fn == "scal":
        return getattr(blas, pre + "scal")(case["alpha"], x.copy(), n=n, incx=incx)
    if fn == "sscal_r":
        return getattr(blas, {"c": "csscal", "z": "zdscal"}[kind])(case["alpha"], x.copy(), n=n, incx=incx)
    if fn in ("dotu", "dotc"):
        name = pre + "dot" if kind in "sd" else pre + fn
        return np.atleast_1d(np.asarray(getattr(blas, name)(x, y, n=n, incx=incx, incy=incy), np.complex128))
    if fn == "asum":
        name = {"s": "sasum", "d": "dasum", "c": "scasum", "z": "dzasum"}[kind]
        return np.array([getattr(blas, name)(x, n=n, incx=incx)], np.float64)
    if fn == "nrm2":
        name = {"s": "snrm2", "d": "dnrm2", "c": "scnrm2", "z": "dznrm2"}[kind]
        return np.array([getattr(blas, name)(x, n=n, incx=incx)], np.float64)
    if fn == "iamax":
        return np.array([getattr(blas, "i" + pre + "amax")(x, n=n, incx=incx)], np.int64)
    if fn == "rot":
        c, s = fx.rot_cs(case)
        name = {"s": "srot", "d": "drot", "c": "csrot", "z": "zdrot"}[kind]
        xo, yo = getattr(blas, name)(x.copy(), y.copy(), c, s, n=n, incx=incx, incy=incy)
        return np.concatenate([xo, yo])
    if fn == "rotm":
        p = np.asarray(case["param"], x.dtype)
        xo, yo = getattr(blas, pre + "rotm")(x.copy(), y.copy(), p, n=n, incx=incx, incy=incy)
        return np.concatenate([xo, yo])
    raise ValueError(fn)


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
    # ---- double and complex level 1 (tests/level1/*.rs fixture ramps)
    for ci, case in enumerate(fx.L1_CASES):
        g[f"l1_c{ci}"] = l1_reference(case)
    for ci, case in enumerate(fx.L1_S_CASES):
        g[f"l1s_c{ci}"] = l1_reference(case)
    for ci, case in enumerate(fx.L1_EDGE_CASES):
        # BLAS's i?amax reports -1 for n = 0; the reference returns 0
        # (isamax.rs:43-151)
        g[f"l1e_c{ci}"] = (np.array([0], np.int64) if case["fn"] == "iamax" and case["n"] == 0
                           else l1_reference(case))
    for ci, (a, b) in enumerate(fx.ROTG_CASES):
        for kind in "sd":
            c, s = getattr(blas, kind + "rotg")(a, b)
            g[f"rotg_{kind}{ci}"] = np.array([c, s], np.float64)
    for ci, (kind, d1, d2, x1, y1) in enumerate(fx.ROTMG_CASES):
        g[f"rotmg_c{ci}"] = np.asarray(getattr(blas, kind + "rotmg")(d1, d2, x1, y1), np.float64)
    # ---- SSYMV / CHEMV (uplo 0 upper, 1 lower), y at fx.sample_index positions
    for si, (n, lda, strides) in enumerate(fx.SYMV_SHAPES):
        A = logical(fx.symv_matrix(n, lda), n, n, lda)
        for (incx, incy) in strides:
            x, y0 = fx.symv_x("s", n, incx), fx.symv_y("s", n, incy)
            for uplo in (0, 1):
                for ci, (alpha, beta) in enumerate(fx.SYMV_COEFFS):
                    r = blas.ssymv(alpha, A, x, beta=beta, y=y0.copy(), incx=incx, incy=incy, lower=uplo)
                    g[f"ssymv_s{si}_{incx}{incy}_u{uplo}_c{ci}"] = S(np.asarray(r, np.float32)[::incy][:n])
    for ci, (uplo, n, lda, alpha, beta, a, x, y0) in enumerate(fx.symv_garbage_cases()):
        r = blas.ssymv(alpha, logical(a, n, n, lda), x, beta=beta, y=y0.copy(), lower=uplo)
        g[f"ssymv_tri{ci}"] = S(np.asarray(r, np.float32))
    for si, (n, lda, strides) in enumerate(fx.HEMV_SHAPES):
        A = logical(fx.hemv_matrix(n, lda), n, n, lda)
        for (incx, incy) in strides:
            x, y0 = fx.hemv_x(n, incx), fx.hemv_y(n, incy)
            for uplo in (0, 1):
                for ci, (alpha, beta) in enumerate(fx.HEMV_COEFFS):
                    r = blas.chemv(alpha, A, x, beta=beta, y=y0.copy(), incx=incx, incy=incy, lower=uplo)
                    g[f"chemv_s{si}_{incx}{incy}_u{uplo}_c{ci}"] = S(np.asarray(r, np.complex64)[::incy][:n])
    for ci, (uplo, n, lda, alpha, beta, a, x, y0) in enumerate(fx.hemv_garbage_cases()):
        r = blas.chemv(alpha, logical(a, n, n, lda), x, beta=beta, y=y0.copy(), lower=uplo)
        g[f"chemv_tri{ci}"] = S(np.asarray(r, np.complex64))
    # ---- STRMV (trans 0 N, 1 T, 2 C; CORAL diag 0 = unit, 1 = non-unit)
    for si, (n, lda, incs) in enumerate(fx.TRMV_SHAPES):
        for uplo in (0, 1):
            for diag in (0, 1):
                A = logical(fx.trmv_matrix(n, lda, uplo, diag), n, n, lda)
                for inc in incs:
                    x = fx.trmv_x(n, inc)
                    for trans in (0, 1, 2):
                        r = blas.strmv(A, x.copy(), incx=inc, lower=uplo, trans=trans,
                                       diag=1 if diag == 0 else 0)
                        g[f"strmv_s{si}_u{uplo}_i{inc}_t{trans}_d{diag}"] = S(np.asarray(r, np.float32)[::inc][:n])
    # ---- SGER / SSYR / SSYR2: the logical matrix at fixed positions
    for ci, (m, n, lda, incx, incy, alpha, gx, gy) in enumerate(fx.GER_CASES):
        A = logical(fx.ger_matrix(m, n, lda), m, n, lda)
        x, y = fx.ramp32(m, incx, gx)[::incx], fx.ramp32(n, incy, gy)[::incy]
        r = np.asarray(blas.sger(alpha, x, y, a=A.copy()), np.float32)
        ri, cj = fx.sample_positions(m, n)
        g[f"sger_c{ci}"] = r[ri, cj]
    for ci, (uplo, n, lda, incx, alpha, gx) in enumerate(fx.SYR_CASES):
        A = logical(fx.syr_matrix(n, lda), n, n, lda)
        x = fx.ramp32(n, incx, gx)
        r = np.asarray(blas.ssyr(alpha, x, lower=uplo, incx=incx, n=n, a=A.copy()), np.float32)
        ri, cj = fx.sample_positions(n, n)
        g[f"ssyr_c{ci}"] = r[ri, cj]
    for ci, (uplo, n, lda, incx, incy, alpha, gx, gy) in enumerate(fx.SYR2_CASES):
        A = logical(fx.syr_matrix(n, lda), n, n, lda)
        x, y = fx.ramp32(n, incx, gx), fx.ramp32(n, incy, gy)
        r = np.asarray(blas.ssyr2(alpha, x, y, lower=uplo, incx=incx, incy=incy, n=n, a=A.copy()),
                       np.float32)
        ri, cj = fx.sample_positions(n, n)
        g[f"ssyr2_c{ci}"] = r[ri, cj]
    # ---- d/c/z GEMV (trans 0 N, 1 T, 2 C)
    for kind, (ops, coeffs, shapes, _, _) in fx.GEMV_DCZ.items():
        for si, (m, n, lda, strides) in enumerate(shapes):
            A = logical(fx.gemv_matrix_k(kind, m, n, lda), m, n, lda)
            for (incx, incy) in strides:
                for trans in ops:
                    xl, yl = (n, m) if trans == 0 else (m, n)
                    x, y0 = fx.gemv_x_k(kind, xl, incx), fx.gemv_y_k(kind, yl, incy)
                    for ci, (alpha, beta) in enumerate(coeffs):
                        r = getattr(blas, kind + "gemv")(alpha, A, x, beta=beta, y=y0.copy(), incx=incx,
                                                         incy=incy, trans=trans)
                        g[f"{kind}gemv_s{si}_{incx}{incy}_t{trans}_c{ci}"] = S(np.asarray(r)[::incy][:yl])
    # ---- DSYMV / ZHEMV
    for kind, name, coeffs, shapes, mat, xg, yg, garbage in (
            ("d", "dsymv", fx.SYMV_COEFFS, fx.SYMV_SHAPES, lambda n, l: fx.symv_matrix(n, l, "d"),
             lambda n, i: fx.symv_x("d", n, i), lambda n, i: fx.symv_y("d", n, i), fx.symv_garbage_cases("d")),
            ("z", "zhemv", fx.ZHEMV_COEFFS, fx.HEMV_SHAPES, lambda n, l: fx.hemv_matrix(n, l, "z"),
             lambda n, i: fx.hemv_x(n, i, "z"), lambda n, i: fx.hemv_y(n, i, "z"), fx.hemv_garbage_cases("z"))):
        for si, (n, lda, strides) in enumerate(shapes):
            A = logical(mat(n, lda), n, n, lda)
            for (incx, incy) in strides:
                x, y0 = xg(n, incx), yg(n, incy)
                for uplo in (0, 1):
                    for ci, (alpha, beta) in enumerate(coeffs):
                        r = getattr(blas, name)(alpha, A, x, beta=beta, y=y0.copy(), incx=incx, incy=incy,
                                                lower=uplo)
                        g[f"{name}_s{si}_{incx}{incy}_u{uplo}_c{ci}"] = S(np.asarray(r)[::incy][:n])
        for ci, (uplo, n, lda, alpha, beta, a, x, y0) in enumerate(garbage):
            r = getattr(blas, name)(alpha, logical(a, n, n, lda), x, beta=beta, y=y0.copy(), lower=uplo)
            g[f"{name}_tri{ci}"] = S(np.asarray(r))
    # ---- d/c/z TRMV and TRSV (CORAL diag 0 = unit, 1 = non-unit)
    for fam, table, mat, xg in (("trmv", fx.TRMV_DCZ, fx.trmv_matrix_k, fx.trmv_x_k),
                                ("trsv", fx.TRSV_DCZ, fx.trsv_matrix_k, fx.trsv_x_k)):
        for kind, (ops, shapes, _, _) in table.items():
            for si, (n, lda, incs) in enumerate(shapes):
                for uplo in (0, 1):
                    for diag in (0, 1):
                        A = logical(mat(kind, n, lda, uplo, diag), n, n, lda)
                        for inc in incs:
                            x = xg(kind, n, inc)
                            for trans in ops:
                                r = getattr(blas, kind + fam)(A, x.copy(), incx=inc, lower=uplo, trans=trans,
                                                              diag=1 if diag == 0 else 0)
                                g[f"{kind}{fam}_s{si}_u{uplo}_i{inc}_t{trans}_d{diag}"] = S(np.asarray(r)[::inc][:n])
    # ---- d/c/z rank updates: the logical matrix at 512 fixed positions
    for ci, (m, n, lda, incx, incy, alpha, gx, gy) in enumerate(fx.GER_CASES):
        A = logical(fx.cm_k("d", m, n, lda, lambda R, i, j: R(0.1) + i * R(0.5) + j * R(0.25)), m, n, lda)
        x, y = fx.rank_vec("d", m, incx, gx)[::incx], fx.rank_vec("d", n, incy, gy)[::incy]
        r = np.asarray(blas.dger(alpha, x, y, a=A.copy()))
        ri, cj = fx.sample_positions(m, n, 512)
        g[f"dger_c{ci}"] = r[ri, cj]
    for ci, (uplo, n, lda, incx, alpha, gx) in enumerate(fx.SYR_CASES):
        A = logical(fx.syr_matrix(n, lda, "d"), n, n, lda)
        r = np.asarray(blas.dsyr(alpha, fx.rank_vec("d", n, incx, gx), lower=uplo, incx=incx, n=n, a=A.copy()))
        ri, cj = fx.sample_positions(n, n, 512)
        g[f"dsyr_c{ci}"] = r[ri, cj]
    for ci, (uplo, n, lda, incx, incy, alpha, gx, gy) in enumerate(fx.SYR2_CASES):
        A = logical(fx.syr_matrix(n, lda, "d"), n, n, lda)
        r = np.asarray(blas.dsyr2(alpha, fx.rank_vec("d", n, incx, gx), fx.rank_vec("d", n, incy, gy), lower=uplo,
                                  incx=incx, incy=incy, n=n, a=A.copy()))
        ri, cj = fx.sample_positions(n, n, 512)
        g[f"dsyr2_c{ci}"] = r[ri, cj]
    for kind in "cz":
        for ci, (m, n, lda, incx, incy, au, ac, gx, gy) in enumerate(fx.CGER_CASES):
            A = logical(fx.gemv_matrix_k(kind, m, n, lda), m, n, lda)
            x, y = fx.rank_vec(kind, m, incx, gx)[::incx], fx.rank_vec(kind, n, incy, gy)[::incy]
            ri, cj = fx.sample_positions(m, n, 512)
            for conj, alpha in ((0, au), (1, ac)):
                fn = getattr(blas, kind + ("gerc" if conj else "geru"))
                r = np.asarray(fn(alpha, x, y, a=A.copy()))
                g[f"{kind}ger_c{ci}_j{conj}"] = r[ri, cj]
        for ci, (uplo, n, lda, incx, alpha, gx) in enumerate(fx.HER_CASES):
            A = logical(fx.hemv_matrix(n, lda, kind), n, n, lda)
            r = np.asarray(getattr(blas, kind + "her")(alpha, fx.rank_vec(kind, n, incx, gx), lower=uplo, incx=incx,
                                                      n=n, a=A.copy()))
            ri, cj = fx.sample_positions(n, n, 512)
            g[f"{kind}her_c{ci}"] = r[ri, cj]
        for ci, (uplo, n, lda, incx, incy, alpha, gx, gy) in enumerate(fx.HER2_CASES):
            A = logical(fx.hemv_matrix(n, lda, kind), n, n, lda)
            r = np.asarray(getattr(blas, kind + "her2")(alpha, fx.rank_vec(kind, n, incx, gx),
                                                       fx.rank_vec(kind, n, incy, gy), lower=uplo, incx=incx,
                                                       incy=incy, n=n, a=A.copy()))
            ri, cj = fx.sample_positions(n, n, 512)
            g[f"{kind}her2_c{ci}"] = r[ri, cj]
    # ---- d/c/z GEMM over every fixture shape: C at fixed positions
    for kind in "dcz":
        for si, (m, n, k, lda_n, lda_t, ldb_n, ldb_t, ldc) in enumerate(fx.GEMM_SHAPES):
            ri, cj = fx.sample_positions(m, n, 64)
            for ci, ((op_a, op_b), (alpha, beta)) in enumerate(fx.gemm_cases_k(kind)):
                lda = lda_n if op_a == 0 else lda_t
                ldb = ldb_n if op_b == 0 else ldb_t
                a, b, c = fx.gemm_operands_k(kind, op_a, op_b, m, n, k, lda, ldb, ldc)
                A = logical(a, *((m, k) if op_a == 0 else (k, m)), lda)
                B = logical(b, *((k, n) if op_b == 0 else (n, k)), ldb)
                r = getattr(blas, kind + "gemm")(alpha, A, B, beta=beta, c=logical(c, m, n, ldc).copy(),
                                                 trans_a=op_a, trans_b=op_b)
                g[f"{kind}gemm_s{si}_c{ci}"] = np.asarray(r)[ri, cj]
    # ---- rank updates applied twice (the reference's run_accumulate_twice)
    ar = fx.ACC_REAL
    for kind in "sd":
        m, n = ar["m"], ar["n"]
        R = np.float32 if kind == "s" else np.float64
        A = logical(fx.cm_k(kind, m, n, m, lambda R_, i, j: R_(0.1) + i * R_(0.5) + j * R_(0.25)), m, n, m)
        for t, (xg, yg) in enumerate(((ar["x1"], ar["y1"]), (ar["x2"], ar["y2"]))):
            A = getattr(blas, kind + "ger")(ar["alpha"][t], fx.rank_vec(kind, m, 1, xg), fx.rank_vec(kind, n, 1, yg),
                                            a=np.asarray(A, R).copy())
        g[f"{kind}ger_acc"] = np.asarray(A, R).ravel(order="F")
        S_ = logical(fx.syr_matrix(m, m, kind), m, m, m)
        S2 = S_.copy()
        for t, (xg, yg) in enumerate(((ar["x1"], ar["y1"]), (ar["x2"], ar["y2"]))):
            S_ = getattr(blas, kind + "syr")(ar["alpha"][t], fx.rank_vec(kind, m, 1, xg), lower=0, a=np.asarray(S_, R).copy())
            S2 = getattr(blas, kind + "syr2")(ar["alpha"][t], fx.rank_vec(kind, m, 1, xg), fx.rank_vec(kind, m, 1, yg),
                                              lower=0, a=np.asarray(S2, R).copy())
        g[f"{kind}syr_acc"] = np.asarray(S_, R).ravel(order="F")
        g[f"{kind}syr2_acc"] = np.asarray(S2, R).ravel(order="F")
    ac, ah, ah2 = fx.ACC_CGER, fx.ACC_HER, fx.ACC_HER2
    for kind in "cz":
        m, n = ac["m"], ac["n"]
        for conj in (0, 1):
            A = logical(fx.gemv_matrix_k(kind, m, n, m), m, n, m)
            fn = getattr(blas, kind + ("gerc" if conj else "geru"))
            for t, (xg, yg) in enumerate(((ac["x1"], ac["y1"]), (ac["x2"], ac["y2"]))):
                A = fn(ac["alpha"][conj][t], fx.rank_vec(kind, m, 1, xg), fx.rank_vec(kind, n, 1, yg), a=A.copy())
            g[f"{kind}ger_acc_j{conj}"] = np.asarray(A).ravel(order="F")
        n = ah["n"]
        H = logical(fx.hemv_matrix(n, n, kind), n, n, n)
        for t, xg in enumerate((ah["x1"], ah["x2"])):
            H = getattr(blas, kind + "her")(ah["alpha"][t], fx.rank_vec(kind, n, 1, xg), lower=0, a=H.copy())
        g[f"{kind}her_acc"] = np.asarray(H).ravel(order="F")
        n = ah2["n"]
        H = logical(fx.hemv_matrix(n, n, kind), n, n, n)
        for t, (xg, yg) in enumerate(((ah2["x1"], ah2["y1"]), (ah2["x2"], ah2["y2"]))):
            H = getattr(blas, kind + "her2")(ah2["alpha"][t], fx.rank_vec(kind, n, 1, xg), fx.rank_vec(kind, n, 1, yg),
                                             lower=0, a=H.copy())
        g[f"{kind}her2_acc"] = np.asarray(H).ravel(order="F")
    # ---- STRSV on the reference's own unit-diagonal matrices, and the
    # triangular files' single-case tests
    for si, (n, lda, incs) in enumerate(fx.TRSV_SHAPES):
        for uplo in (0, 1):
            A = logical(fx.trsv_matrix_k("s", n, lda, uplo, 0), n, n, lda)
            for inc in incs:
                x = fx.trsv_x_k("s", n, inc)
                for trans in (0, 1):
                    r = blas.strsv(A, x.copy(), incx=inc, lower=uplo, trans=trans, diag=1)
                    g[f"strsv_unit_s{si}_u{uplo}_i{inc}_t{trans}"] = S(np.asarray(r, np.float32)[::inc][:n])
    for kind in "sdcz":
        for name, uplo, trans, diag, n, lda, a, x in fx.tri_special_cases(kind, True):
            r = getattr(blas, kind + "trsv")(logical(a, n, n, lda), x.copy(), lower=uplo, trans=trans,
                                             diag=1 if diag == 0 else 0)
            g[f"{kind}trsv_sp_{name}"] = S(np.asarray(r))
    for kind in "sd":
        for name, uplo, trans, diag, n, lda, a, x in fx.tri_special_cases(kind, False):
            r = getattr(blas, kind + "trmv")(logical(a, n, n, lda), x.copy(), lower=uplo, trans=trans,
                                             diag=1 if diag == 0 else 0)
            g[f"{kind}trmv_sp_{name}"] = S(np.asarray(r))
    # ---- SGEMM on the larger fixture shapes (128^3 and the k = 15 panels)
    for si in range(3, len(fx.GEMM_SHAPES)):
        m, n, k, lda_n, lda_t, ldb_n, ldb_t, ldc = fx.GEMM_SHAPES[si]
        ri, cj = fx.sample_positions(m, n, 64)
        for (op_a, op_b) in [(0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (0, 2)]:
            lda = lda_n if op_a == 0 else lda_t
            ldb = ldb_n if op_b == 0 else ldb_t
            a, b, c = fx.gemm_operands(op_a, op_b, m, n, k, lda, ldb, ldc)
            A = logical(a, *((m, k) if op_a == 0 else (k, m)), lda)
            B = logical(b, *((k, n) if op_b == 0 else (n, k)), ldb)
            for ci, (alpha, beta) in enumerate(fx.GEMM_ALPHA_BETA):
                r = blas.sgemm(alpha, A, B, beta=beta, c=logical(c, m, n, ldc).copy(), trans_a=int(op_a != 0),
                               trans_b=int(op_b != 0))
                g[f"sgemm_big_s{si}_{op_a}{op_b}_c{ci}"] = np.asarray(r, np.float32)[ri, cj]
    np.savez_compressed(OUT, **g)
    print(f"wrote {len(g)} arrays to {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
