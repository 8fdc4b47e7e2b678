"""CPU oracle for CORAL's BLAS semantics -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline arm may
import this package, and only as the checker (or, for ``port_*``, as the
timed reference CPU path).  The coral_b200 product never imports it.

Wraps oracle/_build/liboracle.so (built from oracle.c by oracle/Makefile or
:func:`build`).  Functions take numpy arrays.  Parity is pinned by
tests/test_oracle_golden.py against the reference's known-answer doctests,
its planted-maximum isamax cases, the closed-form fixtures of its test suite
and scipy's OpenBLAS (the CBLAS class of oracle the reference's own tests
link), stored as fixtures in tests/golden/.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build() -> str:
    """Compiles oracle.c with its Makefile; returns the library path."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or (
                os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "oracle.c"))):
            build()
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_sz = C.c_size_t
_i = C.c_int


def _declare(L: C.CDLL) -> None:
    L.or_saxpy_exact.argtypes = [_sz, C.c_float, _fp, _sz, _fp, _sz]
    L.or_sscal_exact.argtypes = [_sz, C.c_float, _fp, _sz]
    L.or_scopy_exact.argtypes = [_sz, _fp, _sz, _fp, _sz]
    L.or_sswap_exact.argtypes = [_sz, _fp, _sz, _fp, _sz]
    L.or_isamax_exact.argtypes = [_sz, _fp, _sz]
    L.or_isamax_exact.restype = _sz
    L.or_sdot_f64.argtypes = [_sz, _fp, _sz, _fp, _sz]
    L.or_sdot_f64.restype = C.c_double
    L.or_snrm2_f64.argtypes = [_sz, _fp, _sz]
    L.or_snrm2_f64.restype = C.c_double
    L.or_sgemv_f64.argtypes = [_i, _sz, _sz, C.c_float, _fp, _sz, _fp, _sz, C.c_float, _fp, _sz, _dp]
    L.or_ssymv_f64.argtypes = [_i, _sz, C.c_float, _fp, _sz, _fp, _sz, C.c_float, _fp, _sz, _dp]
    L.or_chemv_f64.argtypes = [_i, _sz, _fp, _fp, _sz, _fp, _sz, _fp, _fp, _sz, _dp]
    L.or_dgemv_f64.argtypes = [_i, _sz, _sz, C.c_double, _dp, _sz, _dp, _sz, C.c_double, _dp, _sz, _dp]
    L.or_cgemv_f64.argtypes = [_i, _sz, _sz, _fp, _fp, _sz, _fp, _sz, _fp, _fp, _sz, _dp]
    L.or_zgemv_f64.argtypes = [_i, _sz, _sz, _dp, _dp, _sz, _dp, _sz, _dp, _dp, _sz, _dp]
    L.or_dsymv_f64.argtypes = [_i, _sz, C.c_double, _dp, _sz, _dp, _sz, C.c_double, _dp, _sz, _dp]
    L.or_zhemv_f64.argtypes = [_i, _sz, _dp, _dp, _sz, _dp, _sz, _dp, _dp, _sz, _dp]
    L.or_dtrmv_f64.argtypes = [_i, _i, _i, _sz, _dp, _sz, _dp, _sz, _dp]
    L.or_ctrmv_f64.argtypes = [_i, _i, _i, _sz, _fp, _sz, _fp, _sz, _dp]
    L.or_ztrmv_f64.argtypes = [_i, _i, _i, _sz, _dp, _sz, _dp, _sz, _dp]
    L.or_dger_f64.argtypes = [_sz, _sz, C.c_double, _dp, _sz, _dp, _sz, _dp, _sz]
    L.or_cger_f64.argtypes = [_i, _sz, _sz, _fp, _fp, _sz, _fp, _sz, _dp, _sz]
    L.or_zger_f64.argtypes = [_i, _sz, _sz, _dp, _dp, _sz, _dp, _sz, _dp, _sz]
    L.or_dsyr_f64.argtypes = [_i, _sz, C.c_double, _dp, _sz, _dp, _sz, _i, _dp, _sz]
    L.or_cher_f64.argtypes = [_i, _sz, _fp, _fp, _sz, _fp, _sz, _i, _dp, _sz]
    L.or_zher_f64.argtypes = [_i, _sz, _dp, _dp, _sz, _dp, _sz, _i, _dp, _sz]
    L.or_dtrsv_f64.argtypes = [_i, _i, _i, _sz, _dp, _sz, _dp, _sz, _dp]
    L.or_ctrsv_f64.argtypes = [_i, _i, _i, _sz, _fp, _sz, _fp, _sz, _dp]
    L.or_ztrsv_f64.argtypes = [_i, _i, _i, _sz, _dp, _sz, _dp, _sz, _dp]
    L.or_strsv_f64.argtypes = [_i, _i, _i, _sz, _fp, _sz, _fp, _sz, _dp]
    L.or_strmv_f64.argtypes = [_i, _i, _i, _sz, _fp, _sz, _fp, _sz, _dp]
    L.or_sger_exact.argtypes = [_sz, _sz, C.c_float, _fp, _sz, _fp, _sz, _fp, _sz]
    L.or_ssyr_exact.argtypes = [_i, _sz, C.c_float, _fp, _sz, _fp, _sz]
    L.or_ssyr2_exact.argtypes = [_i, _sz, C.c_float, _fp, _sz, _fp, _sz, _fp, _sz]
    L.or_gemm_sample.argtypes = [_i, _i, _i, _i, _sz, _sz, _sz, _dp, C.c_void_p, _sz, C.c_void_p,
                                 _sz, _dp, C.c_void_p, _sz, _sz, C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int64), _dp, _dp]
    L.port_sgemm_nn.argtypes = [_sz, _sz, _sz, C.c_float, _fp, _sz, _fp, _sz, C.c_float, _fp, _sz]
    L.port_sgemv_n.argtypes = [_sz, _sz, C.c_float, _fp, _sz, _fp, C.c_float, _fp]
    L.port_sgemv_t.argtypes = [_sz, _sz, C.c_float, _fp, _sz, _fp, C.c_float, _fp]
    L.port_sdot.argtypes = [_sz, _fp, _fp]
    L.port_sdot.restype = C.c_float
    _vp = C.c_void_p
    L.or_axpy_exact.argtypes = [_i, _sz, _dp, _vp, _sz, _vp, _sz]
    L.or_scal_exact.argtypes = [_i, _sz, _dp, _vp, _sz]
    L.or_rot_exact.argtypes = [_i, _sz, _vp, _sz, _vp, _sz, C.c_double, C.c_double]
    L.or_rotm_exact.argtypes = [_i, _sz, _vp, _sz, _vp, _sz, _dp]
    L.or_rotg_exact.argtypes = [_i, _dp]
    L.or_rotmg_exact.argtypes = [_i, _dp, _dp]
    L.or_iamax_exact.argtypes = [_i, _sz, _vp, _sz]
    L.or_iamax_exact.restype = _sz
    L.or_dot_f64.argtypes = [_i, _i, _sz, _vp, _sz, _vp, _sz, _dp]
    L.or_asum_f64.argtypes = [_i, _sz, _vp, _sz]
    L.or_asum_f64.restype = C.c_double
    L.or_nrm2_f64.argtypes = [_i, _sz, _vp, _sz]
    L.or_nrm2_f64.restype = C.c_double


def _f(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(_fp)


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


# ---- level 1 -----------------------------------------------------------------
def saxpy(n, alpha, x, incx, y, incy):
    """In-place on a copy of y; returns it (bit-exact restatement)."""
    y = np.array(y, dtype=np.float32, copy=True)
    lib().or_saxpy_exact(n, alpha, _f(x), incx, _f(y), incy)
    return y


def sscal(n, alpha, x, incx):
    x = np.array(x, dtype=np.float32, copy=True)
    lib().or_sscal_exact(n, alpha, _f(x), incx)
    return x


def scopy(n, x, incx, y, incy):
    y = np.array(y, dtype=np.float32, copy=True)
    lib().or_scopy_exact(n, _f(x), incx, _f(y), incy)
    return y


def sswap(n, x, incx, y, incy):
    x = np.array(x, dtype=np.float32, copy=True)
    y = np.array(y, dtype=np.float32, copy=True)
    lib().or_sswap_exact(n, _f(x), incx, _f(y), incy)
    return x, y


def isamax(n, x, incx) -> int:
    return int(lib().or_isamax_exact(n, _f(x), incx))


def sdot(n, x, incx, y, incy) -> float:
    return float(lib().or_sdot_f64(n, _f(x), incx, _f(y), incy))


def snrm2(n, x, incx) -> float:
    return float(lib().or_snrm2_f64(n, _f(x), incx))


# ---- double and complex level 1 ----------------------------------------------
# kind letters: s float32, d float64, c complex64, z complex128 (numpy arrays
# of those dtypes, increments in elements).
_KIND = {"s": (0, np.float32), "d": (1, np.float64), "c": (2, np.complex64), "z": (3, np.complex128)}


def _vec(kind, a, copy=False):
    dt = _KIND[kind][1]
    a = np.array(a, dtype=dt, copy=True) if copy else np.ascontiguousarray(a, dt)
    return a, C.c_void_p(a.ctypes.data)


def axpy(kind, n, alpha, x, incx, y, incy):
    """s/d/c/z axpy (bit-exact restatement) on a copy of y; returns it."""
    if kind == "s":
        return saxpy(n, float(np.float32(alpha)), x, incx, y, incy)
    al = np.array([complex(alpha).real, complex(alpha).imag], np.float64)
    x, px = _vec(kind, x)
    y, py = _vec(kind, y, copy=True)
    lib().or_axpy_exact(_KIND[kind][0], n, _d(al), px, incx, py, incy)
    return y


def scal(kind, n, alpha, x, incx, real_alpha=False):
    """s/d/c/z scal, or csscal / zdscal with real_alpha (bit-exact); returns a copy."""
    if kind == "s":
        return sscal(n, float(np.float32(alpha)), x, incx)
    al = np.array([complex(alpha).real, complex(alpha).imag], np.float64)
    x, px = _vec(kind, x, copy=True)
    k = _KIND[kind][0]
    if real_alpha:
        k = 4 if kind == "c" else 5
    lib().or_scal_exact(k, n, _d(al), px, incx)
    return x


def copy(n, x, incx, y, incy):
    """Any dtype: y[i*incy] = x[i*incx]; returns a copy of y."""
    y = np.array(y, copy=True)
    if n:
        y[: (n - 1) * incy + 1: incy] = x[: (n - 1) * incx + 1: incx]
    return y


def swap(n, x, incx, y, incy):
    x = np.array(x, copy=True)
    y = np.array(y, copy=True)
    if n:
        sx, sy = slice(0, (n - 1) * incx + 1, incx), slice(0, (n - 1) * incy + 1, incy)
        t = x[sx].copy()
        x[sx] = y[sy]
        y[sy] = t
    return x, y


def rot(kind, n, x, incx, y, incy, c, s):
    """srot / drot / csrot / zdrot (bit-exact); returns (x', y') copies."""
    x, px = _vec(kind, x, copy=True)
    y, py = _vec(kind, y, copy=True)
    lib().or_rot_exact(_KIND[kind][0], n, px, incx, py, incy, float(c), float(s))
    return x, y


def rotm(kind, n, x, incx, y, incy, param):
    """srotm / drotm (bit-exact); returns (x', y') copies."""
    p = np.asarray(param, np.float64)
    x, px = _vec(kind, x, copy=True)
    y, py = _vec(kind, y, copy=True)
    lib().or_rotm_exact(_KIND[kind][0], n, px, incx, py, incy, _d(p))
    return x, y


def rotg(kind, a, b):
    """srotg / drotg: returns (r, z, c, s) in the routine's precision."""
    v = np.array([a, b, 0, 0], np.float64)
    lib().or_rotg_exact(int(kind == "d"), _d(v))
    return tuple(float(t) for t in v)


def rotmg(kind, d1, d2, x1, y1):
    """srotmg / drotmg: returns (d1, d2, x1, param)."""
    v = np.array([d1, d2, x1, y1], np.float64)
    p = np.zeros(5, np.float64)
    lib().or_rotmg_exact(int(kind == "d"), _d(v), _d(p))
    return float(v[0]), float(v[1]), float(v[2]), [float(t) for t in p]


def iamax(kind, n, x, incx) -> int:
    if kind == "s":
        return isamax(n, x, incx)
    x, px = _vec(kind, x)
    return int(lib().or_iamax_exact(_KIND[kind][0], n, px, incx))


def dot(kind, conj, n, x, incx, y, incy) -> complex:
    """ddot / cdotu / cdotc / zdotu / zdotc in double-double (complex result)."""
    x, px = _vec(kind, x)
    y, py = _vec(kind, y)
    out = np.zeros(2, np.float64)
    lib().or_dot_f64(_KIND[kind][0], int(conj), n, px, incx, py, incy, _d(out))
    return complex(out[0], out[1])


def asum(kind, n, x, incx) -> float:
    x, px = _vec(kind, x)
    return float(lib().or_asum_f64(_KIND[kind][0], n, px, incx))


def nrm2(kind, n, x, incx) -> float:
    x, px = _vec(kind, x)
    return float(lib().or_nrm2_f64(_KIND[kind][0], n, px, incx))


# ---- level 2 -----------------------------------------------------------------
def sgemv(trans, m, n, alpha, a, lda, x, incx, beta, y, incy) -> np.ndarray:
    """Returns op(A)-product result y (float64, contiguous length of y)."""
    ylen = n if trans else m
    out = np.zeros(max(ylen, 1), np.float64)
    lib().or_sgemv_f64(trans, m, n, alpha, _f(a), lda, _f(x), incx, beta, _f(y), incy, _d(out))
    return out[:ylen]


def dgemv(trans, m, n, alpha, a, lda, x, incx, beta, y, incy) -> np.ndarray:
    """dgemv result y (float64, contiguous length of y)."""
    ylen = n if trans else m
    out = np.zeros(max(ylen, 1), np.float64)
    lib().or_dgemv_f64(trans, m, n, C.c_double(alpha), _d(np.ascontiguousarray(a, np.float64)), lda,
                       _d(np.ascontiguousarray(x, np.float64)), incx, C.c_double(beta),
                       _d(np.ascontiguousarray(y, np.float64)), incy, _d(out))
    return out[:ylen]


def cgemv(trans, m, n, alpha, a, lda, x, incx, beta, y, incy) -> np.ndarray:
    """cgemv result y as complex128 (inputs complex64 or interleaved float32)."""
    ylen = n if trans else m
    out = np.zeros(2 * max(ylen, 1), np.float64)
    al = np.array([complex(alpha).real, complex(alpha).imag], np.float32)
    be = np.array([complex(beta).real, complex(beta).imag], np.float32)
    f = lambda v: _f(np.ascontiguousarray(v, np.complex64).view(np.float32))  # noqa: E731
    lib().or_cgemv_f64(trans, m, n, _f(al), f(a), lda, f(x), incx, _f(be), f(y), incy, _d(out))
    return out.view(np.complex128)[:ylen]


def zgemv(trans, m, n, alpha, a, lda, x, incx, beta, y, incy) -> np.ndarray:
    """zgemv result y as complex128."""
    ylen = n if trans else m
    out = np.zeros(2 * max(ylen, 1), np.float64)
    al = np.array([complex(alpha).real, complex(alpha).imag], np.float64)
    be = np.array([complex(beta).real, complex(beta).imag], np.float64)
    f = lambda v: _d(np.ascontiguousarray(v, np.complex128).view(np.float64))  # noqa: E731
    lib().or_zgemv_f64(trans, m, n, _d(al), f(a), lda, f(x), incx, _d(be), f(y), incy, _d(out))
    return out.view(np.complex128)[:ylen]


def ssymv(uplo, n, alpha, a, lda, x, incx, beta, y, incy) -> np.ndarray:
    out = np.zeros(max(n, 1), np.float64)
    lib().or_ssymv_f64(uplo, n, alpha, _f(a), lda, _f(x), incx, beta, _f(y), incy, _d(out))
    return out[:n]


def chemv(uplo, n, alpha, a, lda, x, incx, beta, y, incy) -> np.ndarray:
    out = np.zeros(max(2 * n, 2), np.float64)
    al = np.asarray(alpha, np.float32)
    be = np.asarray(beta, np.float32)
    lib().or_chemv_f64(uplo, n, _f(al), _f(a), lda, _f(x), incx, _f(be), _f(y), incy, _d(out))
    return out[:2 * n]


def strsv(uplo, trans, diag, n, a, lda, x, incx) -> np.ndarray:
    out = np.zeros(max(n, 1), np.float64)
    lib().or_strsv_f64(uplo, trans, diag, n, _f(a), lda, _f(x), incx, _d(out))
    return out[:n]


def _c64f(v):
    return _f(np.ascontiguousarray(v, np.complex64).view(np.float32))


def _c128d(v):
    return _d(np.ascontiguousarray(v, np.complex128).view(np.float64))


def dsymv(uplo, n, alpha, a, lda, x, incx, beta, y, incy) -> np.ndarray:
    out = np.zeros(max(n, 1), np.float64)
    f = lambda v: _d(np.ascontiguousarray(v, np.float64))  # noqa: E731
    lib().or_dsymv_f64(uplo, n, C.c_double(alpha), f(a), lda, f(x), incx, C.c_double(beta), f(y), incy,
                       _d(out))
    return out[:n]


def zhemv(uplo, n, alpha, a, lda, x, incx, beta, y, incy) -> np.ndarray:
    """zhemv result as complex128."""
    out = np.zeros(2 * max(n, 1), np.float64)
    al = np.array([complex(alpha).real, complex(alpha).imag], np.float64)
    be = np.array([complex(beta).real, complex(beta).imag], np.float64)
    lib().or_zhemv_f64(uplo, n, _d(al), _c128d(a), lda, _c128d(x), incx, _d(be), _c128d(y), incy, _d(out))
    return out.view(np.complex128)[:n]


def dtrmv(uplo, trans, diag, n, a, lda, x, incx) -> np.ndarray:
    out = np.zeros(max(n, 1), np.float64)
    f = lambda v: _d(np.ascontiguousarray(v, np.float64))  # noqa: E731
    lib().or_dtrmv_f64(uplo, trans, diag, n, f(a), lda, f(x), incx, _d(out))
    return out[:n]


def ctrmv(uplo, trans, diag, n, a, lda, x, incx) -> np.ndarray:
    out = np.zeros(2 * max(n, 1), np.float64)
    lib().or_ctrmv_f64(uplo, trans, diag, n, _c64f(a), lda, _c64f(x), incx, _d(out))
    return out.view(np.complex128)[:n]


def ztrmv(uplo, trans, diag, n, a, lda, x, incx) -> np.ndarray:
    out = np.zeros(2 * max(n, 1), np.float64)
    lib().or_ztrmv_f64(uplo, trans, diag, n, _c128d(a), lda, _c128d(x), incx, _d(out))
    return out.view(np.complex128)[:n]


def dger(m, n, alpha, x, incx, y, incy, a, lda) -> np.ndarray:
    """dger: returns the updated A (float64)."""
    a = np.array(a, dtype=np.float64, copy=True)
    f = lambda v: _d(np.ascontiguousarray(v, np.float64))  # noqa: E731
    lib().or_dger_f64(m, n, C.c_double(alpha), f(x), incx, f(y), incy, _d(a), lda)
    return a


def gerc_u(kind, conj, m, n, alpha, x, incx, y, incy, a, lda) -> np.ndarray:
    """c/z geru (conj = 0) / gerc (conj = 1): returns the updated A as complex128."""
    a = np.array(a, dtype=np.complex128, copy=True)
    if kind == "c":
        al = np.array([complex(alpha).real, complex(alpha).imag], np.float32)
        lib().or_cger_f64(conj, m, n, _f(al), _c64f(x), incx, _c64f(y), incy, _d(a.view(np.float64)), lda)
    else:
        al = np.array([complex(alpha).real, complex(alpha).imag], np.float64)
        lib().or_zger_f64(conj, m, n, _d(al), _c128d(x), incx, _c128d(y), incy, _d(a.view(np.float64)), lda)
    return a


def dsyr(uplo, n, alpha, x, incx, a, lda, y=None, incy=1) -> np.ndarray:
    """dsyr (y None) or dsyr2: returns the updated A (float64)."""
    a = np.array(a, dtype=np.float64, copy=True)
    f = lambda v: _d(np.ascontiguousarray(v, np.float64))  # noqa: E731
    two = y is not None
    lib().or_dsyr_f64(uplo, n, C.c_double(alpha), f(x), incx, f(y if two else x), incy if two else incx,
                      int(two), _d(a), lda)
    return a


def her(kind, uplo, n, alpha, x, incx, a, lda, y=None, incy=1) -> np.ndarray:
    """c/z her (y None; real alpha) or her2: returns the updated A as complex128."""
    a = np.array(a, dtype=np.complex128, copy=True)
    two = y is not None
    yy = y if two else x
    if kind == "c":
        al = np.array([complex(alpha).real, complex(alpha).imag], np.float32)
        lib().or_cher_f64(uplo, n, _f(al), _c64f(x), incx, _c64f(yy), incy if two else incx, int(two),
                          _d(a.view(np.float64)), lda)
    else:
        al = np.array([complex(alpha).real, complex(alpha).imag], np.float64)
        lib().or_zher_f64(uplo, n, _d(al), _c128d(x), incx, _c128d(yy), incy if two else incx, int(two),
                          _d(a.view(np.float64)), lda)
    return a


def trsv_dcz(kind, uplo, trans, diag, n, a, lda, x, incx) -> np.ndarray:
    """d/c/z TRSV solution (float64 or complex128), by long-double substitution."""
    if kind == "d":
        out = np.zeros(max(n, 1), np.float64)
        f = lambda v: _d(np.ascontiguousarray(v, np.float64))  # noqa: E731
        lib().or_dtrsv_f64(uplo, trans, diag, n, f(a), lda, f(x), incx, _d(out))
        return out[:n]
    out = np.zeros(2 * max(n, 1), np.float64)
    if kind == "c":
        lib().or_ctrsv_f64(uplo, trans, diag, n, _c64f(a), lda, _c64f(x), incx, _d(out))
    else:
        lib().or_ztrsv_f64(uplo, trans, diag, n, _c128d(a), lda, _c128d(x), incx, _d(out))
    return out.view(np.complex128)[:n]


def strmv(uplo, trans, diag, n, a, lda, x, incx) -> np.ndarray:
    out = np.zeros(max(n, 1), np.float64)
    lib().or_strmv_f64(uplo, trans, diag, n, _f(a), lda, _f(x), incx, _d(out))
    return out[:n]


def sger(m, n, alpha, x, incx, y, incy, a, lda) -> np.ndarray:
    a = np.array(a, dtype=np.float32, copy=True)
    lib().or_sger_exact(m, n, alpha, _f(x), incx, _f(y), incy, _f(a), lda)
    return a


def ssyr(uplo, n, alpha, x, incx, a, lda) -> np.ndarray:
    a = np.array(a, dtype=np.float32, copy=True)
    lib().or_ssyr_exact(uplo, n, alpha, _f(x), incx, _f(a), lda)
    return a


def ssyr2(uplo, n, alpha, x, incx, y, incy, a, lda) -> np.ndarray:
    a = np.array(a, dtype=np.float32, copy=True)
    lib().or_ssyr2_exact(uplo, n, alpha, _f(x), incx, _f(y), incy, _f(a), lda)
    return a


# ---- level 3 -----------------------------------------------------------------
def gemm_sample(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, rows, cols):
    """Double-double values of selected entries of alpha*op(A)op(B) + beta*C.

    Arrays are flat column-major buffers of float32/float64 (real) or
    complex64/complex128 (complex).  Returns (values, absbound): values is
    complex128 for complex inputs else float64; absbound is
    |alpha|*(|op(A)||op(B)|)_ij + |beta||C_ij| for component-wise errors.
    """
    cplx = np.iscomplexobj(a)
    dbl = a.dtype in (np.float64, np.complex128)
    rows = np.ascontiguousarray(rows, np.int64)
    cols = np.ascontiguousarray(cols, np.int64)
    cnt = rows.size
    out = np.zeros(2 * max(cnt, 1), np.float64)
    absb = np.zeros(max(cnt, 1), np.float64)
    al = np.array([np.real(alpha), np.imag(alpha)], np.float64)
    be = np.array([np.real(beta), np.imag(beta)], np.float64)
    p = lambda arr: np.ascontiguousarray(arr).ctypes.data_as(C.c_void_p)  # noqa: E731
    keep = [np.ascontiguousarray(x) for x in (a, b, c)]
    lib().or_gemm_sample(int(dbl), int(cplx), op_a, op_b, m, n, k, _d(al), p(keep[0]), lda,
                         p(keep[1]), ldb, _d(be), p(keep[2]), ldc, cnt,
                         rows.ctypes.data_as(C.POINTER(C.c_int64)),
                         cols.ctypes.data_as(C.POINTER(C.c_int64)), _d(out), _d(absb))
    vals = out[:2 * cnt].reshape(cnt, 2)
    if cplx:
        return vals[:, 0] + 1j * vals[:, 1], absb[:cnt]
    return vals[:, 0].copy(), absb[:cnt]


def gemm_full(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """Every entry of C (column-major m x n, as a 2-D array [m, n])."""
    ii, jj = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
    vals, absb = gemm_sample(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                             ii.ravel(), jj.ravel())
    return vals.reshape(m, n), absb.reshape(m, n)


# ---- CORAL CPU algorithm restatements (timed as the reference CPU path) ------
def port_sgemm_nn(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    lib().port_sgemm_nn(m, n, k, alpha, _f(a), lda, _f(b), ldb, beta, _f(c), ldc)


def port_sgemv(trans, m, n, alpha, a, lda, x, beta, y):
    fn = lib().port_sgemv_t if trans else lib().port_sgemv_n
    fn(m, n, alpha, _f(a), lda, _f(x), beta, _f(y))


def port_sdot(n, x, y) -> float:
    return float(lib().port_sdot(n, _f(x), _f(y)))
