"""Pins the CPU oracle against the reference's known answers and fixtures.

Known answers: the sgemm and cgemm doctests (coral-aarch64/src/level3/
sgemm.rs:36-81, cgemm.rs:36-96) and the planted-maximum isamax cases
(tests/level1/iamax_tests.rs:79-170).  Fixtures: the closed-form cases of
tests/level3/sgemm_tests.rs, tests/level2/{s,d,c,z}gemv, {s,d}symv,
{c,z}hemv, {s,d,c,z}trsv, {s,d,c,z}trmv, {s,d}ger, {c,z}ger, {s,d}syr,
{s,d}syr2, {c,z}her and {c,z}her2_tests.rs and the level-1 tests, whose
expected outputs were computed by
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


# ---- double and complex level 1 ------------------------------------------------
def oracle_l1(case) -> np.ndarray:
    """The oracle's result for one fx.L1_CASES entry, shaped like the golden
    entry (updated vectors concatenated, or the scalar)."""
    kind, n, fn = case["kind"], case["n"], case["fn"]
    x, y = fx.l1_vectors(case)
    incx, incy = case["incx"], case.get("incy", 1)
    if fn == "axpy":
        return oracle.axpy(kind, n, case["alpha"], x, incx, y, incy)
    if fn == "scal":
        return oracle.scal(kind, n, case["alpha"], x, incx)
    if fn == "sscal_r":
        return oracle.scal(kind, n, case["alpha"], x, incx, real_alpha=True)
    if fn in ("dotu", "dotc"):
        return np.array([oracle.dot(kind, fn == "dotc", n, x, incx, y, incy)])
    if fn == "asum":
        return np.array([oracle.asum(kind, n, x, incx)])
    if fn == "nrm2":
        return np.array([oracle.nrm2(kind, n, x, incx)])
    if fn == "iamax":
        return np.array([oracle.iamax(kind, n, x, incx)])
    if fn == "rot":
        c, s = fx.rot_cs(case)
        return np.concatenate(oracle.rot(kind, n, x, incx, y, incy, c, s))
    if fn == "rotm":
        return np.concatenate(oracle.rotm(kind, n, x, incx, y, incy, case["param"]))
    raise ValueError(fn)


# the reference tests' tolerances: dot_tests.rs:176-179, the other level-1
# test files' RTOL/ATOL (asum_tests.rs:106-109, rot_tests.rs:80-83, ...)
def l1_tol(case):
    if case["kind"] in "sc":
        return (4e-6, 4e-6) if case["fn"].startswith("dot") else (1e-6, 1e-6)
    return 1e-12, 1e-12


@pytest.mark.parametrize("key,case", [(f"l1_c{i}", c) for i, c in enumerate(fx.L1_CASES)] +
                         [(f"l1s_c{i}", c) for i, c in enumerate(fx.L1_S_CASES)] +
                         [(f"l1e_c{i}", c) for i, c in enumerate(fx.L1_EDGE_CASES)])
def test_l1_dcz_fixtures(golden, key, case):
    got, want = oracle_l1(case), golden[key]
    if case["fn"] == "iamax":
        assert int(got[0]) == int(want[0]), case["src"]
        return
    rtol, atol = l1_tol(case)
    got = np.asarray(got, np.complex128)
    want = np.asarray(want, np.complex128)
    assert got.shape == want.shape
    d = np.abs(got - want)
    assert (d <= atol + rtol * np.maximum(np.abs(got), np.abs(want))).all(), (case["src"], d.max())


@pytest.mark.parametrize("kind", "sd")
@pytest.mark.parametrize("ci", range(len(fx.ROTG_CASES)))
def test_rotg_fixtures(golden, kind, ci):
    a, b = fx.ROTG_CASES[ci]
    r, z, c, s = oracle.rotg(kind, a, b)
    tol = 1e-6 if kind == "s" else 1e-12
    np.testing.assert_allclose([c, s], golden[f"rotg_{kind}{ci}"], rtol=tol, atol=tol)
    # r = c a + s b and [c s; -s c] [a; b] = [r; 0]
    assert abs(r - (c * a + s * b)) <= 4 * tol * max(1.0, abs(r))
    assert abs(-s * a + c * b) <= 4 * tol * max(1.0, abs(r))


@pytest.mark.parametrize("ci", range(len(fx.ROTMG_CASES)))
def test_rotmg_fixtures(golden, ci):
    kind, d1, d2, x1, y1 = fx.ROTMG_CASES[ci]
    _, _, _, param = oracle.rotmg(kind, d1, d2, x1, y1)
    tol = 1e-6 if kind == "s" else 1e-12
    want = golden[f"rotmg_c{ci}"]
    assert param[0] == want[0]
    # only the entries the flag makes meaningful (rotmg.rs param packing)
    used = {-1.0: [1, 2, 3, 4], 0.0: [2, 3], 1.0: [1, 4]}.get(param[0], [])
    np.testing.assert_allclose(np.array(param)[used], want[used], rtol=tol, atol=tol)


def test_l1_dcz_rounding_paths():
    """Unit-stride body fused, tail and strided paths rounded per product."""
    rng = np.random.default_rng(11)
    n = 11
    x = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(np.complex64)
    y = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(np.complex64)
    a = np.complex64(0.3 - 0.7j)
    got = oracle.axpy("c", n, a, x, 1, y, 1)
    f32 = np.float32
    for i in range(n):
        xr, xi, yr, yi = f32(x[i].real), f32(x[i].imag), f32(y[i].real), f32(y[i].imag)
        ar, ai = f32(a.real), f32(a.imag)
        if i < 8:   # fused: exact product-sums rounded once per step
            r = f32(np.float64(ar) * xr + yr)
            r = f32(-np.float64(ai) * xi + r)
            m = f32(np.float64(ar) * xi + yi)
            m = f32(np.float64(ai) * xr + m)
        else:
            r = yr + (ar * xr - ai * xi)
            m = yi + (ar * xi + ai * xr)
        assert got[i] == np.complex64(complex(r, m)), i
    # idamax / icamax / izamax: first index, NaN never wins, all NaN -> 0
    v = np.array([np.nan, -3.0, 3.0, np.nan, -3.0])
    assert oracle.iamax("d", 5, v, 1) == 1
    c = np.array([1 + 2j, np.nan, -2 - 1j, 3 + 0j], np.complex64)
    assert oracle.iamax("c", 4, c, 1) == 0
    assert oracle.iamax("z", 3, np.full(3, np.nan, np.complex128), 1) == 0
    # rotm flag -2 and n == 0 leave the vectors alone
    xd, yd = rng.uniform(-1, 1, 5), rng.uniform(-1, 1, 5)
    xo, yo = oracle.rotm("d", 5, xd, 1, yd, 1, [-2, 1, 2, 3, 4])
    np.testing.assert_array_equal(xo, xd)
    np.testing.assert_array_equal(yo, yd)


# ---- symmetric / Hermitian matrix-vector, triangular multiply, rank updates ----
def _S(v):
    """The positions of a result vector that the golden file stores."""
    v = np.asarray(v)
    return v[fx.sample_index(v.size)]


def test_ssymv_fixtures(golden):
    """ssymv_tests.rs:155-249: every shape, stride pair, uplo and (alpha,
    beta) at the reference's 1e-5 / 1e-5 (ssymv_tests.rs:152-153)."""
    from conftest import allclose_ref
    for si, (n, lda, strides) in enumerate(fx.SYMV_SHAPES):
        a = fx.symv_matrix(n, lda)
        for (incx, incy) in strides:
            x, y0 = fx.symv_x("s", n, incx), fx.symv_y("s", n, incy)
            for uplo in (0, 1):
                for ci, (alpha, beta) in enumerate(fx.SYMV_COEFFS):
                    got = oracle.ssymv(uplo, n, alpha, a, lda, x, incx, beta, y0, incy)
                    allclose_ref(_S(got), golden[f"ssymv_s{si}_{incx}{incy}_u{uplo}_c{ci}"], 1e-5, 1e-5)


def test_ssymv_reads_only_the_stored_triangle(golden):
    """ssymv_tests.rs:287-378: NaN in the unstored triangle never reaches y."""
    from conftest import allclose_ref
    for ci, (uplo, n, lda, alpha, beta, a, x, y0) in enumerate(fx.symv_garbage_cases()):
        got = oracle.ssymv(uplo, n, alpha, a, lda, x, 1, beta, y0, 1)
        assert np.isfinite(got).all()
        allclose_ref(_S(got), golden[f"ssymv_tri{ci}"], 1e-5, 1e-5)


def test_ssymv_upper_equals_lower():
    """ssymv_tests.rs:251-285: on a full symmetric matrix both triangles give
    the same y."""
    from conftest import allclose_ref
    n = 513
    a = fx.symv_matrix(n, n)
    x = fx.strided(n, 1, lambda k: fx.f32(-0.07) + fx.f32(0.013) * k)
    y0 = fx.strided(n, 1, lambda k: fx.f32(0.02) - fx.f32(0.004) * k)
    up = oracle.ssymv(0, n, 1.123, a, n, x, 1, -0.321, y0, 1)
    lo = oracle.ssymv(1, n, 1.123, a, n, x, 1, -0.321, y0, 1)
    allclose_ref(up, lo, 1e-5, 1e-5)


def _pair(v):
    return np.array([complex(v).real, complex(v).imag], np.float32)


def test_chemv_fixtures(golden):
    """chemv_tests.rs:194-299 at the reference's 1e-5 / 1e-6
    (chemv_tests.rs:190-191), real and imaginary parts separately."""
    from conftest import allclose_ref
    for si, (n, lda, strides) in enumerate(fx.HEMV_SHAPES):
        a = fx.hemv_matrix(n, lda).view(np.float32)
        for (incx, incy) in strides:
            x, y0 = fx.hemv_x(n, incx).view(np.float32), fx.hemv_y(n, incy).view(np.float32)
            for uplo in (0, 1):
                for ci, (alpha, beta) in enumerate(fx.HEMV_COEFFS):
                    got = oracle.chemv(uplo, n, _pair(alpha), a, lda, x, incx, _pair(beta), y0, incy)
                    want = golden[f"chemv_s{si}_{incx}{incy}_u{uplo}_c{ci}"]
                    allclose_ref(_S(got.view(np.complex128)).view(np.float64), want.view(np.float32), 1e-5, 1e-6)


def test_chemv_reads_only_the_stored_triangle(golden):
    """chemv_tests.rs:360-478: one triangle stored, NaN in the other."""
    from conftest import allclose_ref
    for ci, (uplo, n, lda, alpha, beta, a, x, y0) in enumerate(fx.hemv_garbage_cases()):
        got = oracle.chemv(uplo, n, _pair(alpha), a.view(np.float32), lda, x.view(np.float32), 1,
                           _pair(beta), y0.view(np.float32), 1)
        assert np.isfinite(got).all()
        allclose_ref(_S(got.view(np.complex128)).view(np.float64), golden[f"chemv_tri{ci}"].view(np.float32), 1e-5, 1e-6)


def test_strmv_fixtures(golden):
    """strmv_tests.rs:161-240: both triangles, N/T/C, unit (with a planted
    diagonal that must be ignored) and non-unit, at 1e-5 / 1e-5
    (strmv_tests.rs:154-155)."""
    from conftest import allclose_ref
    for si, (n, lda, incs) in enumerate(fx.TRMV_SHAPES):
        for uplo in (0, 1):
            for diag in (0, 1):
                a = fx.trmv_matrix(n, lda, uplo, diag)
                for inc in incs:
                    x = fx.trmv_x(n, inc)
                    for trans in (0, 1, 2):
                        got = oracle.strmv(uplo, trans, diag, n, a, lda, x, inc)
                        allclose_ref(_S(got), golden[f"strmv_s{si}_u{uplo}_i{inc}_t{trans}_d{diag}"],
                                     1e-5, 1e-5)


def _logical_at(buf, ld, rows, cols):
    return buf[rows + cols * ld]


def test_sger_fixtures(golden):
    """sger_tests.rs:128-197 and the alpha = 0 quick return (:352-356) at
    1e-6 / 1e-6 (sger_tests.rs:82-83); rows past m in each column of a
    padded lda stay as they were."""
    from conftest import allclose_ref
    for ci, (m, n, lda, incx, incy, alpha, gx, gy) in enumerate(fx.GER_CASES):
        a0 = fx.ger_matrix(m, n, lda)
        got = oracle.sger(m, n, alpha, fx.ramp32(m, incx, gx), incx, fx.ramp32(n, incy, gy), incy, a0, lda)
        ri, cj = fx.sample_positions(m, n)
        allclose_ref(_logical_at(got, lda, ri, cj), golden[f"sger_c{ci}"], 1e-6, 1e-6)
        pad = np.ones(lda * n, bool)
        for j in range(n):
            pad[j * lda:j * lda + m] = False
        np.testing.assert_array_equal(got[pad], a0[pad])
        if alpha == 0.0:
            np.testing.assert_array_equal(got, a0)


def _only_triangle_touched(got, a0, n, lda, uplo, bits=np.uint32):
    """ssyr_tests.rs:106-127: the other triangle keeps its bits."""
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    other = (i > j) if uplo == 0 else (i < j)
    idx = (i + j * lda)[other]
    np.testing.assert_array_equal(got[idx].view(bits), a0[idx].view(bits))


def test_ssyr_fixtures(golden):
    """ssyr_tests.rs:132-244 at 1e-6 / 1e-5 (ssyr_tests.rs:129-130), with
    the untouched-triangle check of the small and padded cases."""
    from conftest import allclose_ref
    for ci, (uplo, n, lda, incx, alpha, gx) in enumerate(fx.SYR_CASES):
        a0 = fx.syr_matrix(n, lda)
        got = oracle.ssyr(uplo, n, alpha, fx.ramp32(n, incx, gx), incx, a0, lda)
        ri, cj = fx.sample_positions(n, n)
        allclose_ref(_logical_at(got, lda, ri, cj), golden[f"ssyr_c{ci}"], 1e-6, 1e-5)
        _only_triangle_touched(got, a0, n, lda, uplo)


def test_ssyr2_fixtures(golden):
    """ssyr2_tests.rs:134-245, 350-361 at 1e-6 / 1e-5 (ssyr2_tests.rs:131-132)."""
    from conftest import allclose_ref
    for ci, (uplo, n, lda, incx, incy, alpha, gx, gy) in enumerate(fx.SYR2_CASES):
        a0 = fx.syr_matrix(n, lda)
        got = oracle.ssyr2(uplo, n, alpha, fx.ramp32(n, incx, gx), incx, fx.ramp32(n, incy, gy), incy, a0, lda)
        ri, cj = fx.sample_positions(n, n)
        allclose_ref(_logical_at(got, lda, ri, cj), golden[f"ssyr2_c{ci}"], 1e-6, 1e-5)
        _only_triangle_touched(got, a0, n, lda, uplo)


# ---- d/c/z matrix-vector, symmetric / Hermitian, triangular ----------------------
def _cmp(got, want, rtol, atol):
    """The reference's per-component criterion (real and imaginary parts
    separately for complex results)."""
    from conftest import allclose_ref
    got, want = np.asarray(got), np.asarray(want)
    if np.iscomplexobj(want):
        got = np.asarray(got, np.complex128).view(np.float64)
        want = np.asarray(want, np.complex128).view(np.float64)
    allclose_ref(got, want, rtol, atol)


@pytest.mark.parametrize("kind", ["d", "c", "z"])
def test_gemv_dcz_fixtures(golden, kind):
    """dgemv/cgemv/zgemv_tests.rs: every shape, stride pair, op and (alpha,
    beta) at each file's tolerance."""
    ops, coeffs, shapes, rtol, atol = fx.GEMV_DCZ[kind]
    fn = getattr(oracle, kind + "gemv")
    for si, (m, n, lda, strides) in enumerate(shapes):
        a = fx.gemv_matrix_k(kind, m, n, lda)
        for (incx, incy) in strides:
            for trans in ops:
                xl, yl = (n, m) if trans == 0 else (m, n)
                x, y0 = fx.gemv_x_k(kind, xl, incx), fx.gemv_y_k(kind, yl, incy)
                for ci, (alpha, beta) in enumerate(coeffs):
                    got = fn(trans, m, n, alpha, a, lda, x, incx, beta, y0, incy)
                    _cmp(_S(got), golden[f"{kind}gemv_s{si}_{incx}{incy}_t{trans}_c{ci}"], rtol, atol)


def test_dsymv_fixtures(golden):
    """dsymv_tests.rs:155-378 at 1e-13 / 1e-13 (dsymv_tests.rs:152-153),
    including the NaN-garbage triangle cases."""
    for si, (n, lda, strides) in enumerate(fx.SYMV_SHAPES):
        a = fx.symv_matrix(n, lda, "d")
        for (incx, incy) in strides:
            x, y0 = fx.symv_x("d", n, incx), fx.symv_y("d", n, incy)
            for uplo in (0, 1):
                for ci, (alpha, beta) in enumerate(fx.SYMV_COEFFS):
                    got = oracle.dsymv(uplo, n, alpha, a, lda, x, incx, beta, y0, incy)
                    _cmp(_S(got), golden[f"dsymv_s{si}_{incx}{incy}_u{uplo}_c{ci}"], 1e-13, 1e-13)
    for ci, (uplo, n, lda, alpha, beta, a, x, y0) in enumerate(fx.symv_garbage_cases("d")):
        got = oracle.dsymv(uplo, n, alpha, a, lda, x, 1, beta, y0, 1)
        assert np.isfinite(got).all()
        _cmp(_S(got), golden[f"dsymv_tri{ci}"], 1e-13, 1e-13)


def test_zhemv_fixtures(golden):
    """zhemv_tests.rs:187-478 at 1e-12 / 1e-12 (zhemv_tests.rs:184-185),
    including the NaN-garbage triangle cases."""
    for si, (n, lda, strides) in enumerate(fx.HEMV_SHAPES):
        a = fx.hemv_matrix(n, lda, "z")
        for (incx, incy) in strides:
            x, y0 = fx.hemv_x(n, incx, "z"), fx.hemv_y(n, incy, "z")
            for uplo in (0, 1):
                for ci, (alpha, beta) in enumerate(fx.ZHEMV_COEFFS):
                    got = oracle.zhemv(uplo, n, alpha, a, lda, x, incx, beta, y0, incy)
                    _cmp(_S(got), golden[f"zhemv_s{si}_{incx}{incy}_u{uplo}_c{ci}"], 1e-12, 1e-12)
    for ci, (uplo, n, lda, alpha, beta, a, x, y0) in enumerate(fx.hemv_garbage_cases("z")):
        got = oracle.zhemv(uplo, n, alpha, a, lda, x, 1, beta, y0, 1)
        assert np.isfinite(got).all()
        _cmp(_S(got), golden[f"zhemv_tri{ci}"], 1e-12, 1e-12)


@pytest.mark.parametrize("kind", ["d", "c", "z"])
def test_trmv_dcz_fixtures(golden, kind):
    """dtrmv/ctrmv/ztrmv_tests.rs: both triangles, N/T/C, unit (planted
    diagonal ignored) and non-unit, at each file's tolerance."""
    ops, shapes, rtol, atol = fx.TRMV_DCZ[kind]
    fn = getattr(oracle, kind + "trmv")
    for si, (n, lda, incs) in enumerate(shapes):
        for uplo in (0, 1):
            for diag in (0, 1):
                a = fx.trmv_matrix_k(kind, n, lda, uplo, diag)
                for inc in incs:
                    x = fx.trmv_x_k(kind, n, inc)
                    for trans in ops:
                        got = fn(uplo, trans, diag, n, a, lda, x, inc)
                        _cmp(_S(got), golden[f"{kind}trmv_s{si}_u{uplo}_i{inc}_t{trans}_d{diag}"], rtol, atol)


@pytest.mark.parametrize("kind", ["d", "c", "z"])
def test_trsv_dcz_fixtures(golden, kind):
    """dtrsv/ctrsv/ztrsv_tests.rs: both triangles, every op, unit (planted
    diagonal ignored) and non-unit, padded lda and strides, at each file's
    tolerance."""
    ops, shapes, rtol, atol = fx.TRSV_DCZ[kind]
    for si, (n, lda, incs) in enumerate(shapes):
        for uplo in (0, 1):
            for diag in (0, 1):
                a = fx.trsv_matrix_k(kind, n, lda, uplo, diag)
                for inc in incs:
                    x = fx.trsv_x_k(kind, n, inc)
                    for trans in ops:
                        got = oracle.trsv_dcz(kind, uplo, trans, diag, n, a, lda, x, inc)
                        _cmp(_S(got), golden[f"{kind}trsv_s{si}_u{uplo}_i{inc}_t{trans}_d{diag}"], rtol, atol)


def test_rank_dz_real_fixtures(golden):
    """dger/dsyr/dsyr2_tests.rs: the sger/ssyr/ssyr2 case tables in f64 at
    each file's tolerance; the syr forms leave the other triangle's bits."""
    for ci, (m, n, lda, incx, incy, alpha, gx, gy) in enumerate(fx.GER_CASES):
        a0 = fx.cm_k("d", m, n, lda, lambda R, i, j: R(0.1) + i * R(0.5) + j * R(0.25))
        got = oracle.dger(m, n, alpha, fx.rank_vec("d", m, incx, gx), incx, fx.rank_vec("d", n, incy, gy), incy,
                          a0, lda)
        ri, cj = fx.sample_positions(m, n, 512)
        _cmp(_logical_at(got, lda, ri, cj), golden[f"dger_c{ci}"], *fx.RANK_TOL["dger"])
    for ci, (uplo, n, lda, incx, alpha, gx) in enumerate(fx.SYR_CASES):
        a0 = fx.syr_matrix(n, lda, "d")
        got = oracle.dsyr(uplo, n, alpha, fx.rank_vec("d", n, incx, gx), incx, a0, lda)
        ri, cj = fx.sample_positions(n, n, 512)
        _cmp(_logical_at(got, lda, ri, cj), golden[f"dsyr_c{ci}"], *fx.RANK_TOL["dsyr"])
        _only_triangle_touched(got, a0, n, lda, uplo, np.uint64)
    for ci, (uplo, n, lda, incx, incy, alpha, gx, gy) in enumerate(fx.SYR2_CASES):
        a0 = fx.syr_matrix(n, lda, "d")
        got = oracle.dsyr(uplo, n, alpha, fx.rank_vec("d", n, incx, gx), incx, a0, lda,
                          y=fx.rank_vec("d", n, incy, gy), incy=incy)
        ri, cj = fx.sample_positions(n, n, 512)
        _cmp(_logical_at(got, lda, ri, cj), golden[f"dsyr2_c{ci}"], *fx.RANK_TOL["dsyr2"])
        _only_triangle_touched(got, a0, n, lda, uplo, np.uint64)


@pytest.mark.parametrize("kind", ["c", "z"])
def test_rank_complex_fixtures(golden, kind):
    """cger/zger (geru and gerc), cher/zher and cher2/zher2_tests.rs at each
    file's tolerance; the Hermitian forms leave the other triangle's bits."""
    for ci, (m, n, lda, incx, incy, au, ac, gx, gy) in enumerate(fx.CGER_CASES):
        a0 = fx.gemv_matrix_k(kind, m, n, lda)
        ri, cj = fx.sample_positions(m, n, 512)
        for conj, alpha in ((0, au), (1, ac)):
            got = oracle.gerc_u(kind, conj, m, n, alpha, fx.rank_vec(kind, m, incx, gx), incx,
                                fx.rank_vec(kind, n, incy, gy), incy, a0, lda)
            _cmp(_logical_at(got, lda, ri, cj), golden[f"{kind}ger_c{ci}_j{conj}"], *fx.RANK_TOL[kind + "ger"])
    for ci, (uplo, n, lda, incx, alpha, gx) in enumerate(fx.HER_CASES):
        a0 = fx.hemv_matrix(n, lda, kind)
        got = oracle.her(kind, uplo, n, alpha, fx.rank_vec(kind, n, incx, gx), incx, a0, lda)
        ri, cj = fx.sample_positions(n, n, 512)
        _cmp(_logical_at(got, lda, ri, cj), golden[f"{kind}her_c{ci}"], *fx.RANK_TOL[kind + "her"])
        _herm_other_triangle_kept(got, a0, n, lda, uplo)
    for ci, (uplo, n, lda, incx, incy, alpha, gx, gy) in enumerate(fx.HER2_CASES):
        a0 = fx.hemv_matrix(n, lda, kind)
        got = oracle.her(kind, uplo, n, alpha, fx.rank_vec(kind, n, incx, gx), incx, a0, lda,
                         y=fx.rank_vec(kind, n, incy, gy), incy=incy)
        ri, cj = fx.sample_positions(n, n, 512)
        _cmp(_logical_at(got, lda, ri, cj), golden[f"{kind}her2_c{ci}"], *fx.RANK_TOL[kind + "her2"])
        _herm_other_triangle_kept(got, a0, n, lda, uplo)


def _herm_other_triangle_kept(got, a0, n, lda, uplo):
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    other = (i > j) if uplo == 0 else (i < j)
    idx = (i + j * lda)[other]
    np.testing.assert_array_equal(np.asarray(got)[idx], np.asarray(a0, np.complex128)[idx])


@pytest.mark.parametrize("kind", ["d", "c", "z"])
def test_gemm_dcz_fixtures(golden, kind):
    """dgemm/cgemm/zgemm_tests.rs over every fixture shape (including the
    128^3 and the thin k = 15 panels), every op pair and (alpha, beta) of each
    file, at each file's tolerance (real and imaginary parts separately)."""
    rtol, atol = fx.GEMM_TOL[kind]
    for si, (m, n, k, lda_n, lda_t, ldb_n, ldb_t, ldc) in enumerate(fx.GEMM_SHAPES):
        ri, cj = fx.sample_positions(m, n, 64)
        for ci, ((op_a, op_b), (alpha, beta)) in enumerate(fx.gemm_cases_k(kind)):
            lda = lda_n if op_a == 0 else lda_t
            ldb = ldb_n if op_b == 0 else ldb_t
            a, b, c = fx.gemm_operands_k(kind, op_a, op_b, m, n, k, lda, ldb, ldc)
            got, _ = oracle.gemm_sample(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ri, cj)
            _cmp(got, golden[f"{kind}gemm_s{si}_c{ci}"], rtol, atol)


def test_rank_updates_applied_twice(golden):
    """Each rank-update file's run_accumulate_twice: two updates in a row on
    the same matrix, every entry against BLAS at the file's tolerance."""
    ar = fx.ACC_REAL
    m, n = ar["m"], ar["n"]
    pairs = ((ar["x1"], ar["y1"]), (ar["x2"], ar["y2"]))
    for kind in "sd":
        a = fx.cm_k(kind, m, n, m, lambda R, i, j: R(0.1) + i * R(0.5) + j * R(0.25))
        s1 = fx.syr_matrix(m, m, kind)
        s2 = s1.copy()
        for t, (xg, yg) in enumerate(pairs):
            x, y = fx.rank_vec(kind, m, 1, xg), fx.rank_vec(kind, n, 1, yg)
            xs, ys = x, fx.rank_vec(kind, m, 1, yg)
            if kind == "s":
                a = oracle.sger(m, n, ar["alpha"][t], x, 1, y, 1, a, m)
                s1 = oracle.ssyr(0, m, ar["alpha"][t], xs, 1, s1, m)
                s2 = oracle.ssyr2(0, m, ar["alpha"][t], xs, 1, ys, 1, s2, m)
            else:
                a = oracle.dger(m, n, ar["alpha"][t], x, 1, y, 1, a, m)
                s1 = oracle.dsyr(0, m, ar["alpha"][t], xs, 1, s1, m)
                s2 = oracle.dsyr(0, m, ar["alpha"][t], xs, 1, s2, m, y=ys, incy=1)
        _cmp(a, golden[f"{kind}ger_acc"], *fx.RANK_TOL[kind + "ger"])
        _cmp(s1, golden[f"{kind}syr_acc"], *fx.RANK_TOL[kind + "syr"])
        _cmp(s2, golden[f"{kind}syr2_acc"], *fx.RANK_TOL[kind + "syr2"])
    ac, ah, ah2 = fx.ACC_CGER, fx.ACC_HER, fx.ACC_HER2
    for kind in "cz":
        for conj in (0, 1):
            a = fx.gemv_matrix_k(kind, m, n, m)
            for t, (xg, yg) in enumerate(((ac["x1"], ac["y1"]), (ac["x2"], ac["y2"]))):
                a = oracle.gerc_u(kind, conj, m, n, ac["alpha"][conj][t], fx.rank_vec(kind, m, 1, xg), 1,
                                  fx.rank_vec(kind, n, 1, yg), 1, a, m)
            _cmp(a, golden[f"{kind}ger_acc_j{conj}"], *fx.RANK_TOL[kind + "ger"])
        nh = ah["n"]
        h = fx.hemv_matrix(nh, nh, kind)
        for t, xg in enumerate((ah["x1"], ah["x2"])):
            h = oracle.her(kind, 0, nh, ah["alpha"][t], fx.rank_vec(kind, nh, 1, xg), 1, h, nh)
        _cmp(h, golden[f"{kind}her_acc"], *fx.RANK_TOL[kind + "her"])
        nh = ah2["n"]
        h = fx.hemv_matrix(nh, nh, kind)
        for t, (xg, yg) in enumerate(((ah2["x1"], ah2["y1"]), (ah2["x2"], ah2["y2"]))):
            h = oracle.her(kind, 0, nh, ah2["alpha"][t], fx.rank_vec(kind, nh, 1, xg), 1, h, nh,
                           y=fx.rank_vec(kind, nh, 1, yg), incy=1)
        _cmp(h, golden[f"{kind}her2_acc"], *fx.RANK_TOL[kind + "her2"])


def _mirror(au, al, n, lda, conj, rtol, atol):
    """assert_upper_lower_equal(_c): upper (i, j), i <= j, against lower
    (j, i) -- conjugated for the Hermitian forms."""
    i, j = np.nonzero(np.triu(np.ones((n, n), bool)))
    up = np.asarray(au)[i + j * lda]
    lo = np.asarray(al)[j + i * lda]
    _cmp(up, np.conj(lo) if conj else lo, rtol, atol)


@pytest.mark.parametrize("real,cplx", [("s", "c"), ("d", "z")])
def test_rank_updates_upper_equals_lower(real, cplx):
    """ssyr/ssyr2/cher/cher2_tests.rs run_upper_equals_lower (and the d/z
    files): on a full symmetric / Hermitian matrix the upper and the lower
    update are mirror images."""
    n = 33
    x = fx.rank_vec(real, n, 1, (0.2, 0.005))
    y = fx.rank_vec(real, n, 1, (0.1, 0.004))
    a = fx.syr_matrix(n, n, real)
    if real == "s":
        up, lo = oracle.ssyr(0, n, 0.77, x, 1, a, n), oracle.ssyr(1, n, 0.77, x, 1, a, n)
        up2, lo2 = oracle.ssyr2(0, n, 0.77, x, 1, y, 1, a, n), oracle.ssyr2(1, n, 0.77, x, 1, y, 1, a, n)
    else:
        up, lo = oracle.dsyr(0, n, 0.77, x, 1, a, n), oracle.dsyr(1, n, 0.77, x, 1, a, n)
        up2 = oracle.dsyr(0, n, 0.77, x, 1, a, n, y=y, incy=1)
        lo2 = oracle.dsyr(1, n, 0.77, x, 1, a, n, y=y, incy=1)
    _mirror(up, lo, n, n, False, *fx.RANK_TOL[real + "syr"])
    _mirror(up2, lo2, n, n, False, *fx.RANK_TOL[real + "syr2"])
    nh = 25
    xh = fx.rank_vec(cplx, nh, 1, (0.2, 0.005, -0.04, 0.002))
    h = fx.hemv_matrix(nh, nh, cplx)
    _mirror(oracle.her(cplx, 0, nh, 0.77, xh, 1, h, nh), oracle.her(cplx, 1, nh, 0.77, xh, 1, h, nh), nh, nh, True,
            *fx.RANK_TOL[cplx + "her"])
    x2 = fx.rank_vec(cplx, n, 1, (0.2, 0.005, -0.04, 0.002))
    y2 = fx.rank_vec(cplx, n, 1, (0.1, 0.004, 0.03, -0.001))
    h2 = fx.hemv_matrix(n, n, cplx)
    _mirror(oracle.her(cplx, 0, n, 0.77 + 0.11j, x2, 1, h2, n, y=y2, incy=1),
            oracle.her(cplx, 1, n, 0.77 + 0.11j, x2, 1, h2, n, y=y2, incy=1), n, n, True, *fx.RANK_TOL[cplx + "her2"])


def test_rank_and_trmv_quick_returns():
    """The quick-return cases of sger/ssyr/strmv_tests.rs (m = 0 or n = 0):
    nothing is written."""
    a = np.zeros(5, np.float32)
    np.testing.assert_array_equal(oracle.sger(0, 5, 0.77, np.ones(1, np.float32), 1,
                                              fx.rank_vec("s", 5, 1, (0.2, 0.1)), 1, a, 1), a)
    np.testing.assert_array_equal(oracle.ssyr(0, 0, 0.55, np.zeros(1, np.float32), 1, np.zeros(1, np.float32), 1),
                                  np.zeros(1, np.float32))
    assert oracle.strmv(0, 0, 1, 0, np.zeros(1, np.float32), 1, np.zeros(1, np.float32), 1).size == 0


def test_strsv_reference_unit_matrices(golden):
    """strsv_tests.rs run_all with build_matrix's unit-diagonal matrices
    (make_upper_unit / make_lower_unit with a planted diagonal that a unit
    call must ignore), at 1e-4 (strsv_tests.rs:213-214)."""
    for si, (n, lda, incs) in enumerate(fx.TRSV_SHAPES):
        for uplo in (0, 1):
            a = fx.trsv_matrix_k("s", n, lda, uplo, 0)
            for inc in incs:
                x = fx.trsv_x_k("s", n, inc)
                for trans in (0, 1):
                    got = oracle.strsv(uplo, trans, 0, n, a, lda, x, inc)
                    _cmp(_S(got), golden[f"strsv_unit_s{si}_u{uplo}_i{inc}_t{trans}"], 1e-4, 1e-4)


TRI_TOL = {"strsv": (1e-4, 1e-4), "dtrsv": (1e-12, 1e-12), "ctrsv": (1e-2, 1e-3), "ztrsv": (1e-11, 1e-11),
           "strmv": (1e-5, 1e-5), "dtrmv": (1e-13, 1e-13)}


@pytest.mark.parametrize("kind", ["s", "d", "c", "z"])
def test_triangular_single_cases(golden, kind):
    """lower_transpose_padded (both triangles populated, lda > n),
    unitdiag_upper_notranspose and unitdiag_lower_transpose of
    {s,d,c,z}trsv_tests.rs, padded_lower_transpose of {s,d}trmv_tests.rs,
    and the n = 0 quick returns."""
    for name, uplo, trans, diag, n, lda, a, x in fx.tri_special_cases(kind, True):
        got = (oracle.strsv(uplo, trans, diag, n, a, lda, x, 1) if kind == "s"
               else oracle.trsv_dcz(kind, uplo, trans, diag, n, a, lda, x, 1))
        _cmp(_S(got), golden[f"{kind}trsv_sp_{name}"], *TRI_TOL[kind + "trsv"])
    if kind in "sd":
        for name, uplo, trans, diag, n, lda, a, x in fx.tri_special_cases(kind, False):
            got = getattr(oracle, kind + "trmv")(uplo, trans, diag, n, a, lda, x, 1)
            _cmp(_S(got), golden[f"{kind}trmv_sp_{name}"], *TRI_TOL[kind + "trmv"])
    z = np.zeros(2, fx._DT[kind])
    solve = (oracle.strsv(0, 0, 1, 0, z, 1, z, 1) if kind == "s" else oracle.trsv_dcz(kind, 0, 0, 1, 0, z, 1, z, 1))
    assert solve.size == 0


@pytest.mark.parametrize("si", range(3, len(fx.GEMM_SHAPES)))
def test_sgemm_larger_fixtures(golden, si):
    """sgemm_tests.rs medium_square_all_ops (128^3) and rectangular_all_ops
    (k = 15 panels), C at 64 fixed positions, at the reference's 1e-3
    (sgemm_tests.rs:85-86): at k = 128 the ramps cancel, and OpenBLAS's fp32
    sums then sit about 1.5e-5 from the exact values the oracle gives."""
    m, n, k, lda_n, lda_t, ldb_n, ldb_t, ldc = fx.GEMM_SHAPES[si]
    ri, cj = fx.sample_positions(m, n, 64)
    for (op_a, op_b) in [(0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (0, 2)]:
        lda = lda_n if op_a == 0 else lda_t
        ldb = ldb_n if op_b == 0 else ldb_t
        a, b, c = fx.gemm_operands(op_a, op_b, m, n, k, lda, ldb, ldc)
        for ci, (alpha, beta) in enumerate(fx.GEMM_ALPHA_BETA):
            got, _ = oracle.gemm_sample(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ri, cj)
            _cmp(got, golden[f"sgemm_big_s{si}_{op_a}{op_b}_c{ci}"], 1e-3, 1e-3)


@pytest.mark.parametrize("kind", ["d", "c", "z"])
def test_symv_hemv_upper_equals_lower(kind):
    """dsymv_tests.rs (n = 513) and chemv/zhemv_tests.rs (n = 257)
    upper_equals_lower: on a full symmetric / Hermitian matrix both
    triangles give the same y."""
    if kind == "d":
        n = 513
        a = fx.symv_matrix(n, n, "d")
        x = fx.rvec("d", n, 1, lambda R, k: R(-0.07) + R(0.013) * k)
        y = fx.rvec("d", n, 1, lambda R, k: R(0.02) - R(0.004) * k)
        up = oracle.dsymv(0, n, 1.123, a, n, x, 1, -0.321, y, 1)
        lo = oracle.dsymv(1, n, 1.123, a, n, x, 1, -0.321, y, 1)
        _cmp(up, lo, 1e-13, 1e-13)
        return
    n = 257
    a = fx.hemv_matrix(n, n, kind)
    x = fx.cvec(kind, n, 1, lambda R, k: R(-0.07) + R(0.013) * k, lambda R, k: R(0.015) - R(0.002) * k)
    y = fx.cvec(kind, n, 1, lambda R, k: R(0.02) - R(0.004) * k, lambda R, k: R(-0.01) + R(0.001) * k)
    al, be = 1.123 - 0.321j, -0.321 + 0.777j
    if kind == "c":
        f = lambda u: oracle.chemv(u, n, _pair(al), a.view(np.float32), n, x.view(np.float32), 1,  # noqa: E731
                                   _pair(be), y.view(np.float32), 1)
        _cmp(f(0), f(1), 1e-5, 1e-6)
    else:
        _cmp(oracle.zhemv(0, n, al, a, n, x, 1, be, y, 1), oracle.zhemv(1, n, al, a, n, x, 1, be, y, 1), 1e-12, 1e-12)


@pytest.mark.parametrize("n,incx,incy", [(1024, 1, 1), (777, 3, 2), (0, 1, 1), (1, 5, 7)])
def test_scopy_sswap_bitwise(n, incx, incy):
    """copy_tests.rs / swap_tests.rs (real f32 cases): the strided copy and
    swap move every bit, NaN payloads and -0.0 included; elements between
    the strided positions are untouched."""
    rng = np.random.default_rng(n + incx)
    lx, ly = max((n - 1) * incx + 1, 1), max((n - 1) * incy + 1, 1)
    bits = rng.integers(0, 2**32, lx + ly, dtype=np.uint64).astype(np.uint32)
    bits[::7] = 0x7FC01234       # a NaN with a payload
    bits[3::11] = 0x80000000     # -0.0
    x, y = bits[:lx].view(np.float32).copy(), bits[lx:].view(np.float32).copy()
    want_y = y.copy()
    if n:
        want_y[: (n - 1) * incy + 1: incy] = x[: (n - 1) * incx + 1: incx]
    np.testing.assert_array_equal(oracle.scopy(n, x, incx, y, incy).view(np.uint32), want_y.view(np.uint32))
    sx, sy = oracle.sswap(n, x, incx, y, incy)
    want_x = x.copy()
    if n:
        want_x[: (n - 1) * incx + 1: incx] = y[: (n - 1) * incy + 1: incy]
    np.testing.assert_array_equal(sx.view(np.uint32), want_x.view(np.uint32))
    np.testing.assert_array_equal(sy.view(np.uint32), want_y.view(np.uint32))
