"""CORAL's BLAS API over the B200 engine.

Every function keeps the name, argument order and argument meaning of the
reference routine it replaces (coral-aarch64/src/level{1,2,3}); matrices and
vectors are CUDA tensors (``torch.Tensor`` on an sm_100 device) whose storage
plays the role of the reference's slices/pointers, and work is enqueued on
PyTorch's current stream.  Routines that update in place (``y``, ``x``, ``c``,
``matrix``) update the tensor passed in; routines that return a value in the
reference (``sdot``, ``snrm2``, ``isamax``) return it.

Where the reference would ``debug_assert!`` (bad increments, short buffers,
lda too small) these functions raise :class:`CoralError` carrying the BLAS
argument position, instead of undefined behaviour.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import enum
import threading

from . import _lib


class CoralTranspose(enum.IntEnum):
    """coral-aarch64/src/enums.rs:1-6."""
    NoTranspose = 0
    Transpose = 1
    ConjugateTranspose = 2


class CoralTriangular(enum.IntEnum):
    """coral-aarch64/src/enums.rs:8-12."""
    UpperTriangular = 0
    LowerTriangular = 1


class CoralDiagonal(enum.IntEnum):
    """coral-aarch64/src/enums.rs:14-18."""
    UnitDiagonal = 0
    NonUnitDiagonal = 1


class GemmMode(enum.IntEnum):
    NATIVE = 0
    SPLIT_BF16X3 = 1
    OZAKI_INT8 = 2
    SPLIT_BF16X6 = 3


STATUS = {0: "CORAL_OK", 1: "CORAL_ERR_INVALID_ARG", 2: "CORAL_ERR_CUDA",
          3: "CORAL_ERR_TIMEOUT", 4: "CORAL_ERR_ALLOC", 5: "CORAL_ERR_NOT_SUPPORTED",
          6: "CORAL_ERR_NO_DEVICE"}


class CoralError(RuntimeError):
    def __init__(self, status: int, routine: str, bad_arg: int = 0, detail: str = ""):
        self.status = status
        self.bad_arg = bad_arg
        msg = f"{routine}: {STATUS.get(status, status)}"
        if status == 1:
            msg += f" (argument {bad_arg})"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


class Handle:
    """Owns a coral_handle_t bound to a CUDA stream."""

    def __init__(self):
        self.lib = _lib.load()
        h = C.c_void_p()
        st = self.lib.coral_create(C.byref(h))
        if st != 0:
            raise CoralError(st, "coral_create")
        self.h = h

    def close(self) -> None:
        if self.h:
            self.lib.coral_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bind_current_stream(self) -> None:
        import torch
        self.lib.coral_set_stream(self.h, C.c_void_p(torch.cuda.current_stream().cuda_stream))

    def set_gemm_mode(self, mode: int) -> None:
        self.check(self.lib.coral_set_gemm_mode(self.h, int(mode)), "coral_set_gemm_mode")

    def gemm_mode(self) -> int:
        m = C.c_int()
        self.check(self.lib.coral_get_gemm_mode(self.h, C.byref(m)), "coral_get_gemm_mode")
        return m.value

    def set_pointer_mode(self, mode: int) -> None:
        """0: scalar results to host memory (waits); 1: to device memory (async)."""
        self.check(self.lib.coral_set_pointer_mode(self.h, int(mode)), "coral_set_pointer_mode")

    def set_split_chunk(self, slabs: int) -> None:
        self.check(self.lib.coral_set_split_chunk(self.h, slabs), "coral_set_split_chunk")

    def set_complex_mapping(self, mapping: int) -> None:
        """0: 4M (default), 1: 3M, for coral_cgemm in the split-BF16 modes."""
        self.check(self.lib.coral_set_complex_mapping(self.h, mapping), "coral_set_complex_mapping")

    def set_strip_form(self, form: int) -> None:
        """0: register-streaming SYMV/HEMV/TRMV (default), 1: the TMA-fed single pass when the matrix allows."""
        self.check(self.lib.coral_set_strip_form(self.h, form), "coral_set_strip_form")

    def set_gemm_tile(self, tile_m: int, tile_n: int, split_k: int) -> None:
        """Split-GEMM tile: (128, 128 | 256) one CTA per tile, (256, 256) a CTA pair; zeros: policy."""
        self.check(self.lib.coral_set_gemm_tile(self.h, tile_m, tile_n, split_k), "coral_set_gemm_tile")

    def gemm_tile(self, products: int, op_a: int, op_b: int, m: int, n: int, k: int) -> tuple[int, int, int]:
        """(tile_m, tile_n, split_k) a split GEMM of this shape would use now."""
        tm, tn, sk = C.c_int(), C.c_int(), C.c_int()
        self.check(self.lib.coral_get_gemm_tile(self.h, products, op_a, op_b, m, n, k, C.byref(tm),
                                                C.byref(tn), C.byref(sk)), "coral_get_gemm_tile")
        return tm.value, tn.value, sk.value

    def set_pair_raster(self, group: int) -> None:
        self.check(self.lib.coral_set_pair_raster(self.h, group), "coral_set_pair_raster")

    def set_wait_limit(self, spins: int) -> None:
        self.check(self.lib.coral_set_wait_limit(self.h, spins), "coral_set_wait_limit")

    def set_kernel_timing(self, enable: bool) -> None:
        self.check(self.lib.coral_set_kernel_timing(self.h, int(enable)), "coral_set_kernel_timing")

    def kernel_timing(self) -> tuple[float, int]:
        """(summed ms, launches) of the dominant kernels timed since the last query."""
        ms, n = C.c_double(), C.c_uint64()
        self.check(self.lib.coral_get_kernel_timing(self.h, C.byref(ms), C.byref(n)),
                   "coral_get_kernel_timing")
        return ms.value, n.value

    def sync(self) -> None:
        self.check(self.lib.coral_sync(self.h), "coral_sync")

    def check(self, status: int, routine: str) -> None:
        if status != 0:
            bad = self.lib.coral_last_bad_arg(self.h) if self.h else 0
            detail = (self.lib.coral_last_cuda_error(self.h) or b"").decode() if status == 2 else ""
            raise CoralError(status, routine, bad, detail)

    def call(self, name: str, *args) -> None:
        self.bind_current_stream()
        self.check(getattr(self.lib, name)(self.h, *args), name)


_tls = threading.local()


def handle() -> Handle:
    """This thread's default handle."""
    h = getattr(_tls, "handle", None)
    if h is None:
        h = Handle()
        _tls.handle = h
    return h


def _ptr(t, dtypes, name: str):
    """Device address of tensor `t` (None -> NULL)."""
    if t is None:
        return None
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype not in dtypes:
        raise TypeError(f"{name} has dtype {t.dtype}, expected one of {dtypes}")
    return C.c_void_p(t.data_ptr())


def _f32():
    import torch
    return (torch.float32,)


def _f64():
    import torch
    return (torch.float64,)


def _c64():
    import torch
    return (torch.complex64, torch.float32)


def _c128():
    import torch
    return (torch.complex128, torch.float64)


# ---------------------------------------------------------------- level 1 ----
def sdot(n, x, incx, y, incy) -> float:
    """level1/sdot.rs:42-161."""
    r = C.c_float()
    handle().call("coral_sdot", n, _ptr(x, _f32(), "x"), incx, _ptr(y, _f32(), "y"), incy,
                  C.cast(C.byref(r), C.c_void_p))
    return r.value


def saxpy(n, alpha, x, incx, y, incy) -> None:
    """level1/saxpy.rs:42-131 (y updated in place)."""
    handle().call("coral_saxpy", n, alpha, _ptr(x, _f32(), "x"), incx, _ptr(y, _f32(), "y"), incy)


def snrm2(n, x, incx) -> float:
    """level1/snrm2.rs:45-149."""
    r = C.c_float()
    handle().call("coral_snrm2", n, _ptr(x, _f32(), "x"), incx, C.cast(C.byref(r), C.c_void_p))
    return r.value


def isamax(n, x, incx) -> int:
    """level1/isamax.rs:43-151 (0-based index)."""
    r = C.c_size_t()
    handle().call("coral_isamax", n, _ptr(x, _f32(), "x"), incx, C.cast(C.byref(r), C.c_void_p))
    return r.value


def scopy(n, x, incx, y, incy) -> None:
    """level1/scopy.rs:28-58."""
    handle().call("coral_scopy", n, _ptr(x, _f32(), "x"), incx, _ptr(y, _f32(), "y"), incy)


def sswap(n, x, incx, y, incy) -> None:
    """level1/sswap.rs:35-118."""
    handle().call("coral_sswap", n, _ptr(x, _f32(), "x"), incx, _ptr(y, _f32(), "y"), incy)


def sscal(n, alpha, x, incx) -> None:
    """level1/sscal.rs:30-66."""
    handle().call("coral_sscal", n, alpha, _ptr(x, _f32(), "x"), incx)


# Double and complex level 1: complex vectors are complex64 / complex128
# tensors (or float32 / float64 interleaved), increments in complex elements.
_L1_KIND = {"s": (_f32, C.c_float), "d": (_f64, C.c_double), "c": (_c64, C.c_float), "z": (_c128, C.c_double)}


def _reduce_scalar(name, kind, n, x, incx, out_ctype):
    dt = _L1_KIND[kind][0]
    r = out_ctype()
    handle().call(name, n, _ptr(x, dt(), "x"), incx, C.cast(C.byref(r), C.c_void_p))
    return r.value


def ddot(n, x, incx, y, incy) -> float:
    """level1/ddot.rs:43-163."""
    r = C.c_double()
    handle().call("coral_ddot", n, _ptr(x, _f64(), "x"), incx, _ptr(y, _f64(), "y"), incy,
                  C.cast(C.byref(r), C.c_void_p))
    return r.value


def _cdot(name, kind, n, x, incx, y, incy) -> complex:
    dt, ct = _L1_KIND[kind]
    r = (ct * 2)()
    handle().call(name, n, _ptr(x, dt(), "x"), incx, _ptr(y, dt(), "y"), incy, C.cast(r, C.c_void_p))
    return complex(r[0], r[1])


def cdotu(n, x, incx, y, incy) -> complex:
    """level1/cdotu.rs:46-178: sum x_i y_i."""
    return _cdot("coral_cdotu", "c", n, x, incx, y, incy)


def cdotc(n, x, incx, y, incy) -> complex:
    """level1/cdotc.rs:46-176: sum conj(x_i) y_i."""
    return _cdot("coral_cdotc", "c", n, x, incx, y, incy)


def zdotu(n, x, incx, y, incy) -> complex:
    """level1/zdotu.rs:45-176."""
    return _cdot("coral_zdotu", "z", n, x, incx, y, incy)


def zdotc(n, x, incx, y, incy) -> complex:
    """level1/zdotc.rs:45-175."""
    return _cdot("coral_zdotc", "z", n, x, incx, y, incy)


def sasum(n, x, incx) -> float:
    """level1/sasum.rs:40-107."""
    return _reduce_scalar("coral_sasum", "s", n, x, incx, C.c_float)


def dasum(n, x, incx) -> float:
    """level1/dasum.rs:41-110."""
    return _reduce_scalar("coral_dasum", "d", n, x, incx, C.c_double)


def scasum(n, x, incx) -> float:
    """level1/scasum.rs:40-108: sum |re| + |im|."""
    return _reduce_scalar("coral_scasum", "c", n, x, incx, C.c_float)


def dzasum(n, x, incx) -> float:
    """level1/dzasum.rs:40-111."""
    return _reduce_scalar("coral_dzasum", "z", n, x, incx, C.c_double)


def dnrm2(n, x, incx) -> float:
    """level1/dnrm2.rs:45-152."""
    return _reduce_scalar("coral_dnrm2", "d", n, x, incx, C.c_double)


def scnrm2(n, x, incx) -> float:
    """level1/scnrm2.rs:44-155."""
    return _reduce_scalar("coral_scnrm2", "c", n, x, incx, C.c_float)


def dznrm2(n, x, incx) -> float:
    """level1/dznrm2.rs:43-156."""
    return _reduce_scalar("coral_dznrm2", "z", n, x, incx, C.c_double)


def idamax(n, x, incx) -> int:
    """level1/idamax.rs:43-159 (0-based index)."""
    return _reduce_scalar("coral_idamax", "d", n, x, incx, C.c_size_t)


def icamax(n, x, incx) -> int:
    """level1/icamax.rs:48-166: first max |re| + |im| (0-based)."""
    return _reduce_scalar("coral_icamax", "c", n, x, incx, C.c_size_t)


def izamax(n, x, incx) -> int:
    """level1/izamax.rs:33-163."""
    return _reduce_scalar("coral_izamax", "z", n, x, incx, C.c_size_t)


def daxpy(n, alpha, x, incx, y, incy) -> None:
    """level1/daxpy.rs:42-133."""
    handle().call("coral_daxpy", n, float(alpha), _ptr(x, _f64(), "x"), incx, _ptr(y, _f64(), "y"), incy)


def caxpy(n, alpha, x, incx, y, incy) -> None:
    """level1/caxpy.rs:45-172 (alpha: complex or [re, im])."""
    pa, ka = _pair(_cscalar(alpha), C.c_float)
    handle().call("coral_caxpy", n, pa, _ptr(x, _c64(), "x"), incx, _ptr(y, _c64(), "y"), incy)


def zaxpy(n, alpha, x, incx, y, incy) -> None:
    """level1/zaxpy.rs:44-172."""
    pa, ka = _pair(_cscalar(alpha), C.c_double)
    handle().call("coral_zaxpy", n, pa, _ptr(x, _c128(), "x"), incx, _ptr(y, _c128(), "y"), incy)


def dscal(n, alpha, x, incx) -> None:
    """level1/dscal.rs:30-66."""
    handle().call("coral_dscal", n, float(alpha), _ptr(x, _f64(), "x"), incx)


def cscal(n, alpha, x, incx) -> None:
    """level1/cscal.rs:43-111."""
    pa, ka = _pair(_cscalar(alpha), C.c_float)
    handle().call("coral_cscal", n, pa, _ptr(x, _c64(), "x"), incx)


def zscal(n, alpha, x, incx) -> None:
    """level1/zscal.rs:41-109."""
    pa, ka = _pair(_cscalar(alpha), C.c_double)
    handle().call("coral_zscal", n, pa, _ptr(x, _c128(), "x"), incx)


def csscal(n, alpha, x, incx) -> None:
    """level1/csscal.rs:39-88: real alpha, complex64 x."""
    handle().call("coral_csscal", n, float(alpha), _ptr(x, _c64(), "x"), incx)


def zdscal(n, alpha, x, incx) -> None:
    """level1/zdscal.rs:38-88: real alpha, complex128 x."""
    handle().call("coral_zdscal", n, float(alpha), _ptr(x, _c128(), "x"), incx)


def _xy(name, kind, n, x, incx, y, incy, *extra) -> None:
    dt = _L1_KIND[kind][0]
    handle().call(name, n, _ptr(x, dt(), "x"), incx, _ptr(y, dt(), "y"), incy, *extra)


def dcopy(n, x, incx, y, incy) -> None:
    """level1/dcopy.rs:28-57."""
    _xy("coral_dcopy", "d", n, x, incx, y, incy)


def ccopy(n, x, incx, y, incy) -> None:
    """level1/ccopy.rs:29-58."""
    _xy("coral_ccopy", "c", n, x, incx, y, incy)


def zcopy(n, x, incx, y, incy) -> None:
    """level1/zcopy.rs:28-61."""
    _xy("coral_zcopy", "z", n, x, incx, y, incy)


def dswap(n, x, incx, y, incy) -> None:
    """level1/dswap.rs:35-119."""
    _xy("coral_dswap", "d", n, x, incx, y, incy)


def cswap(n, x, incx, y, incy) -> None:
    """level1/cswap.rs:36-120."""
    _xy("coral_cswap", "c", n, x, incx, y, incy)


def zswap(n, x, incx, y, incy) -> None:
    """level1/zswap.rs:35-120."""
    _xy("coral_zswap", "z", n, x, incx, y, incy)


def srot(n, x, incx, y, incy, c, s) -> None:
    """level1/srot.rs:51-180."""
    _xy("coral_srot", "s", n, x, incx, y, incy, float(c), float(s))


def drot(n, x, incx, y, incy, c, s) -> None:
    """level1/drot.rs:48-178."""
    _xy("coral_drot", "d", n, x, incx, y, incy, float(c), float(s))


def csrot(n, x, incx, y, incy, c, s) -> None:
    """level1/csrot.rs:50-166: real c, s on complex64 vectors."""
    _xy("coral_csrot", "c", n, x, incx, y, incy, float(c), float(s))


def zdrot(n, x, incx, y, incy, c, s) -> None:
    """level1/zdrot.rs:51-166."""
    _xy("coral_zdrot", "z", n, x, incx, y, incy, float(c), float(s))


def srotm(n, x, incx, y, incy, param) -> None:
    """level1/srotm.rs:47-412: param = [flag, h11, h21, h12, h22]."""
    p = (C.c_float * 5)(*[float(v) for v in param])
    _xy("coral_srotm", "s", n, x, incx, y, incy, C.cast(p, C.c_void_p))


def drotm(n, x, incx, y, incy, param) -> None:
    """level1/drotm.rs:47-410."""
    p = (C.c_double * 5)(*[float(v) for v in param])
    _xy("coral_drotm", "d", n, x, incx, y, incy, C.cast(p, C.c_void_p))


def _rotg(name, ct, a, b):
    v = [ct(a), ct(b), ct(), ct()]
    handle().call(name, *[C.cast(C.byref(t), C.c_void_p) for t in v])
    return tuple(t.value for t in v)


def srotg(a, b):
    """level1/srotg.rs:40-75: returns (r, z, c, s) -- the updated a, b and c, s."""
    return _rotg("coral_srotg", C.c_float, a, b)


def drotg(a, b):
    """level1/drotg.rs:40-71: returns (r, z, c, s)."""
    return _rotg("coral_drotg", C.c_double, a, b)


def _rotmg(name, ct, d1, d2, x1, y1):
    v = [ct(d1), ct(d2), ct(x1)]
    p = (ct * 5)()
    handle().call(name, *[C.cast(C.byref(t), C.c_void_p) for t in v], ct(y1), C.cast(p, C.c_void_p))
    return v[0].value, v[1].value, v[2].value, list(p)


def srotmg(d1, d2, x1, y1):
    """level1/srotmg.rs:42-199: returns (d1, d2, x1, param)."""
    return _rotmg("coral_srotmg", C.c_float, d1, d2, x1, y1)


def drotmg(d1, d2, x1, y1):
    """level1/drotmg.rs:41-195: returns (d1, d2, x1, param)."""
    return _rotmg("coral_drotmg", C.c_double, d1, d2, x1, y1)


# ------------------------------------------------------- fused level 1.5 ----
_FUSED_DT = {"s": _f32, "d": _f64, "c": _c64, "z": _c128}


def _axpyf(kind, n_rows, n_cols, x, incx, matrix, lda, y, incy) -> None:
    dt = _FUSED_DT[kind]
    handle().call(f"coral_{kind}axpyf", n_rows, n_cols, _ptr(x, dt(), "x"), incx, _ptr(matrix, dt(), "matrix"),
                  lda, _ptr(y, dt(), "y"), incy)


def _dotf(name, kind, n_rows, n_cols, matrix, lda, x, incx, out) -> None:
    dt = _FUSED_DT[kind]
    handle().call(name, n_rows, n_cols, _ptr(matrix, dt(), "matrix"), lda, _ptr(x, dt(), "x"), incx,
                  _ptr(out, dt(), "out"))


def saxpyf(n_rows, n_cols, x, incx, matrix, lda, y, incy) -> None:
    """level1_special/saxpyf.rs:36-513: y += A x."""
    _axpyf("s", n_rows, n_cols, x, incx, matrix, lda, y, incy)


def daxpyf(n_rows, n_cols, x, incx, matrix, lda, y, incy) -> None:
    """level1_special/daxpyf.rs:45-518."""
    _axpyf("d", n_rows, n_cols, x, incx, matrix, lda, y, incy)


def caxpyf(n_rows, n_cols, x, incx, matrix, lda, y, incy) -> None:
    """level1_special/caxpyf.rs:48-696."""
    _axpyf("c", n_rows, n_cols, x, incx, matrix, lda, y, incy)


def zaxpyf(n_rows, n_cols, x, incx, matrix, lda, y, incy) -> None:
    """level1_special/zaxpyf.rs:49-697."""
    _axpyf("z", n_rows, n_cols, x, incx, matrix, lda, y, incy)


def sdotf(n_rows, n_cols, matrix, lda, x, incx, out) -> None:
    """level1_special/sdotf.rs:37-600: out += A^T x."""
    _dotf("coral_sdotf", "s", n_rows, n_cols, matrix, lda, x, incx, out)


def ddotf(n_rows, n_cols, matrix, lda, x, incx, out) -> None:
    """level1_special/ddotf.rs:37-596."""
    _dotf("coral_ddotf", "d", n_rows, n_cols, matrix, lda, x, incx, out)


def cdotuf(n_rows, n_cols, matrix, lda, x, incx, out) -> None:
    """level1_special/cdotuf.rs:41-764: out += A^T x."""
    _dotf("coral_cdotuf", "c", n_rows, n_cols, matrix, lda, x, incx, out)


def cdotcf(n_rows, n_cols, matrix, lda, x, incx, out) -> None:
    """level1_special/cdotcf.rs:42-765: out += A^H x."""
    _dotf("coral_cdotcf", "c", n_rows, n_cols, matrix, lda, x, incx, out)


def zdotuf(n_rows, n_cols, matrix, lda, x, incx, out) -> None:
    """level1_special/zdotuf.rs:41-665."""
    _dotf("coral_zdotuf", "z", n_rows, n_cols, matrix, lda, x, incx, out)


def zdotcf(n_rows, n_cols, matrix, lda, x, incx, out) -> None:
    """level1_special/zdotcf.rs:41-1000."""
    _dotf("coral_zdotcf", "z", n_rows, n_cols, matrix, lda, x, incx, out)


# ---------------------------------------------------------------- level 2 ----
def sgemv(trans, n_rows, n_cols, alpha, matrix, lda, x, incx, beta, y, incy) -> None:
    """level2/sgemv.rs:63-80."""
    handle().call("coral_sgemv", int(trans), n_rows, n_cols, alpha, _ptr(matrix, _f32(), "matrix"),
                  lda, _ptr(x, _f32(), "x"), incx, beta, _ptr(y, _f32(), "y"), incy)


def dgemv(trans, n_rows, n_cols, alpha, matrix, lda, x, incx, beta, y, incy) -> None:
    """level2/dgemv.rs."""
    handle().call("coral_dgemv", int(trans), n_rows, n_cols, float(alpha), _ptr(matrix, _f64(), "matrix"),
                  lda, _ptr(x, _f64(), "x"), incx, float(beta), _ptr(y, _f64(), "y"), incy)


def _cscalar(z):
    return complex(z[0], z[1]) if isinstance(z, (list, tuple)) else complex(z)


def cgemv(trans, n_rows, n_cols, alpha, matrix, lda, x, incx, beta, y, incy) -> None:
    """level2/cgemv.rs:60-80 (alpha/beta: complex or [re, im])."""
    pa, ka = _pair(_cscalar(alpha), C.c_float)
    pb, kb = _pair(_cscalar(beta), C.c_float)
    handle().call("coral_cgemv", int(trans), n_rows, n_cols, pa, _ptr(matrix, _c64(), "matrix"), lda,
                  _ptr(x, _c64(), "x"), incx, pb, _ptr(y, _c64(), "y"), incy)


def zgemv(trans, n_rows, n_cols, alpha, matrix, lda, x, incx, beta, y, incy) -> None:
    """level2/zgemv.rs (alpha/beta: complex or [re, im])."""
    pa, ka = _pair(_cscalar(alpha), C.c_double)
    pb, kb = _pair(_cscalar(beta), C.c_double)
    handle().call("coral_zgemv", int(trans), n_rows, n_cols, pa, _ptr(matrix, _c128(), "matrix"), lda,
                  _ptr(x, _c128(), "x"), incx, pb, _ptr(y, _c128(), "y"), incy)


def dsymv(uplo, n, alpha, matrix, lda, x, incx, beta, y, incy) -> None:
    """level2/dsymv.rs:99-210."""
    handle().call("coral_dsymv", int(uplo), n, float(alpha), _ptr(matrix, _f64(), "matrix"), lda,
                  _ptr(x, _f64(), "x"), incx, float(beta), _ptr(y, _f64(), "y"), incy)


def zhemv(uplo, n, alpha, matrix, lda, x, incx, beta, y, incy) -> None:
    """level2/zhemv.rs:96-230 (alpha/beta: complex or [re, im])."""
    pa, ka = _pair(_cscalar(alpha), C.c_double)
    pb, kb = _pair(_cscalar(beta), C.c_double)
    handle().call("coral_zhemv", int(uplo), n, pa, _ptr(matrix, _c128(), "matrix"), lda,
                  _ptr(x, _c128(), "x"), incx, pb, _ptr(y, _c128(), "y"), incy)


def dtrmv(uplo, transpose, diagonal, n, matrix, lda, x, incx) -> None:
    """level2/dtrmv.rs (x overwritten with op(A) x)."""
    handle().call("coral_dtrmv", int(uplo), int(transpose), int(diagonal), n,
                  _ptr(matrix, _f64(), "matrix"), lda, _ptr(x, _f64(), "x"), incx)


def ctrmv(uplo, transpose, diagonal, n, matrix, lda, x, incx) -> None:
    """level2/ctrmv.rs:58-72."""
    handle().call("coral_ctrmv", int(uplo), int(transpose), int(diagonal), n,
                  _ptr(matrix, _c64(), "matrix"), lda, _ptr(x, _c64(), "x"), incx)


def ztrmv(uplo, transpose, diagonal, n, matrix, lda, x, incx) -> None:
    """level2/ztrmv.rs."""
    handle().call("coral_ztrmv", int(uplo), int(transpose), int(diagonal), n,
                  _ptr(matrix, _c128(), "matrix"), lda, _ptr(x, _c128(), "x"), incx)


def dger(n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda) -> None:
    """level2/dger.rs."""
    handle().call("coral_dger", n_rows, n_cols, float(alpha), _ptr(x, _f64(), "x"), incx,
                  _ptr(y, _f64(), "y"), incy, _ptr(matrix, _f64(), "matrix"), lda)


def _cger(name, kind, n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda):
    pa, ka = _pair(_cscalar(alpha), C.c_float if kind == "c" else C.c_double)
    dt = _c64() if kind == "c" else _c128()
    handle().call(name, n_rows, n_cols, pa, _ptr(x, dt, "x"), incx, _ptr(y, dt, "y"), incy,
                  _ptr(matrix, dt, "matrix"), lda)


def cgeru(n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda) -> None:
    """level2/cgeru.rs: A += alpha x y^T."""
    _cger("coral_cgeru", "c", n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda)


def cgerc(n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda) -> None:
    """level2/cgerc.rs: A += alpha x y^H."""
    _cger("coral_cgerc", "c", n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda)


def zgeru(n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda) -> None:
    """level2/zgeru.rs."""
    _cger("coral_zgeru", "z", n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda)


def zgerc(n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda) -> None:
    """level2/zgerc.rs."""
    _cger("coral_zgerc", "z", n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda)


def dsyr(uplo, n, alpha, x, incx, matrix, lda) -> None:
    """level2/dsyr.rs."""
    handle().call("coral_dsyr", int(uplo), n, float(alpha), _ptr(x, _f64(), "x"), incx,
                  _ptr(matrix, _f64(), "matrix"), lda)


def dsyr2(uplo, n, alpha, x, incx, y, incy, matrix, lda) -> None:
    """level2/dsyr2.rs."""
    handle().call("coral_dsyr2", int(uplo), n, float(alpha), _ptr(x, _f64(), "x"), incx,
                  _ptr(y, _f64(), "y"), incy, _ptr(matrix, _f64(), "matrix"), lda)


def cher(uplo, n, alpha, x, incx, matrix, lda) -> None:
    """level2/cher.rs (real alpha)."""
    handle().call("coral_cher", int(uplo), n, float(alpha), _ptr(x, _c64(), "x"), incx,
                  _ptr(matrix, _c64(), "matrix"), lda)


def zher(uplo, n, alpha, x, incx, matrix, lda) -> None:
    """level2/zher.rs (real alpha)."""
    handle().call("coral_zher", int(uplo), n, float(alpha), _ptr(x, _c128(), "x"), incx,
                  _ptr(matrix, _c128(), "matrix"), lda)


def _cher2(name, kind, uplo, n, alpha, x, incx, y, incy, matrix, lda):
    pa, ka = _pair(_cscalar(alpha), C.c_float if kind == "c" else C.c_double)
    dt = _c64() if kind == "c" else _c128()
    handle().call(name, int(uplo), n, pa, _ptr(x, dt, "x"), incx, _ptr(y, dt, "y"), incy,
                  _ptr(matrix, dt, "matrix"), lda)


def cher2(uplo, n, alpha, x, incx, y, incy, matrix, lda) -> None:
    """level2/cher2.rs."""
    _cher2("coral_cher2", "c", uplo, n, alpha, x, incx, y, incy, matrix, lda)


def zher2(uplo, n, alpha, x, incx, y, incy, matrix, lda) -> None:
    """level2/zher2.rs."""
    _cher2("coral_zher2", "z", uplo, n, alpha, x, incx, y, incy, matrix, lda)


def dtrsv(uplo, transpose, diagonal, n, matrix, lda, x, incx) -> None:
    """level2/dtrsv.rs (x solved in place)."""
    handle().call("coral_dtrsv", int(uplo), int(transpose), int(diagonal), n,
                  _ptr(matrix, _f64(), "matrix"), lda, _ptr(x, _f64(), "x"), incx)


def ctrsv(uplo, transpose, diagonal, n, matrix, lda, x, incx) -> None:
    """level2/ctrsv.rs (x solved in place)."""
    handle().call("coral_ctrsv", int(uplo), int(transpose), int(diagonal), n,
                  _ptr(matrix, _c64(), "matrix"), lda, _ptr(x, _c64(), "x"), incx)


def ztrsv(uplo, transpose, diagonal, n, matrix, lda, x, incx) -> None:
    """level2/ztrsv.rs (x solved in place)."""
    handle().call("coral_ztrsv", int(uplo), int(transpose), int(diagonal), n,
                  _ptr(matrix, _c128(), "matrix"), lda, _ptr(x, _c128(), "x"), incx)


def ssymv(uplo, n, alpha, matrix, lda, x, incx, beta, y, incy) -> None:
    """level2/ssymv.rs:99-394."""
    handle().call("coral_ssymv", int(uplo), n, alpha, _ptr(matrix, _f32(), "matrix"), lda,
                  _ptr(x, _f32(), "x"), incx, beta, _ptr(y, _f32(), "y"), incy)


def _pair(z, ctype):
    arr = (ctype * 2)(complex(z).real, complex(z).imag)
    return C.cast(arr, C.c_void_p), arr


def chemv(uplo, n, alpha, matrix, lda, x, incx, beta, y, incy) -> None:
    """level2/chemv.rs:96-447 (alpha/beta: complex or [re, im])."""
    if isinstance(alpha, (list, tuple)):
        alpha = complex(alpha[0], alpha[1])
    if isinstance(beta, (list, tuple)):
        beta = complex(beta[0], beta[1])
    pa, ka = _pair(alpha, C.c_float)
    pb, kb = _pair(beta, C.c_float)
    handle().call("coral_chemv", int(uplo), n, pa, _ptr(matrix, _c64(), "matrix"), lda,
                  _ptr(x, _c64(), "x"), incx, pb, _ptr(y, _c64(), "y"), incy)


def strsv(uplo, transpose, diagonal, n, matrix, lda, x, incx) -> None:
    """level2/strsv.rs:60-74 (x solved in place)."""
    handle().call("coral_strsv", int(uplo), int(transpose), int(diagonal), n,
                  _ptr(matrix, _f32(), "matrix"), lda, _ptr(x, _f32(), "x"), incx)


def strmv(uplo, transpose, diagonal, n, matrix, lda, x, incx) -> None:
    """level2/strmv.rs:59-73 (x updated in place)."""
    handle().call("coral_strmv", int(uplo), int(transpose), int(diagonal), n,
                  _ptr(matrix, _f32(), "matrix"), lda, _ptr(x, _f32(), "x"), incx)


def sger(n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda) -> None:
    """level2/sger.rs:68-132."""
    handle().call("coral_sger", n_rows, n_cols, alpha, _ptr(x, _f32(), "x"), incx,
                  _ptr(y, _f32(), "y"), incy, _ptr(matrix, _f32(), "matrix"), lda)


def ssyr(uplo, n, alpha, x, incx, matrix, lda) -> None:
    """level2/ssyr.rs:63-181."""
    handle().call("coral_ssyr", int(uplo), n, alpha, _ptr(x, _f32(), "x"), incx,
                  _ptr(matrix, _f32(), "matrix"), lda)


def ssyr2(uplo, n, alpha, x, incx, y, incy, matrix, lda) -> None:
    """level2/ssyr2.rs:59-197."""
    handle().call("coral_ssyr2", int(uplo), n, alpha, _ptr(x, _f32(), "x"), incx,
                  _ptr(y, _f32(), "y"), incy, _ptr(matrix, _f32(), "matrix"), lda)


# ---------------------------------------------------------------- level 3 ----
def sgemm(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> None:
    """level3/sgemm.rs:106-130; arithmetic per the handle's GEMM mode."""
    handle().call("coral_sgemm", int(op_a), int(op_b), m, n, k, alpha, _ptr(a, _f32(), "a"), lda,
                  _ptr(b, _f32(), "b"), ldb, beta, _ptr(c, _f32(), "c"), ldc)


def dgemm(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> None:
    """level3/dgemm.rs:107."""
    handle().call("coral_dgemm", int(op_a), int(op_b), m, n, k, alpha, _ptr(a, _f64(), "a"), lda,
                  _ptr(b, _f64(), "b"), ldb, beta, _ptr(c, _f64(), "c"), ldc)


def cgemm(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> None:
    """level3/cgemm.rs:127-157 (alpha/beta: complex or [re, im])."""
    if isinstance(alpha, (list, tuple)):
        alpha = complex(alpha[0], alpha[1])
    if isinstance(beta, (list, tuple)):
        beta = complex(beta[0], beta[1])
    pa, ka = _pair(alpha, C.c_float)
    pb, kb = _pair(beta, C.c_float)
    handle().call("coral_cgemm", int(op_a), int(op_b), m, n, k, pa, _ptr(a, _c64(), "a"), lda,
                  _ptr(b, _c64(), "b"), ldb, pb, _ptr(c, _c64(), "c"), ldc)


def zgemm(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> None:
    """level3/zgemm.rs:123 (alpha/beta: complex or [re, im])."""
    if isinstance(alpha, (list, tuple)):
        alpha = complex(alpha[0], alpha[1])
    if isinstance(beta, (list, tuple)):
        beta = complex(beta[0], beta[1])
    pa, ka = _pair(alpha, C.c_double)
    pb, kb = _pair(beta, C.c_double)
    handle().call("coral_zgemm", int(op_a), int(op_b), m, n, k, pa, _ptr(a, _c128(), "a"), lda,
                  _ptr(b, _c128(), "b"), ldb, pb, _ptr(c, _c128(), "c"), ldc)


def set_gemm_mode(mode: int) -> None:
    handle().set_gemm_mode(mode)


def gemm_mode() -> int:
    return handle().gemm_mode()


def set_gemm_tile(tile_m: int, tile_n: int, split_k: int = 0) -> None:
    handle().set_gemm_tile(tile_m, tile_n, split_k)


# ------------------------------------------------------- batched (no reference) --
SGEMM_PROBLEM_DTYPE = None


def sgemm_problem_dtype():
    """numpy dtype matching coral_sgemm_problem_t (80 bytes)."""
    import numpy as np
    return np.dtype([("op_a", "<i4"), ("op_b", "<i4"), ("m", "<i4"), ("n", "<i4"), ("k", "<i4"),
                     ("alpha", "<f4"), ("beta", "<f4"), ("reserved", "<i4"), ("a", "<u8"),
                     ("b", "<u8"), ("c", "<u8"), ("lda", "<i8"), ("ldb", "<i8"), ("ldc", "<i8")])


def strsv_problem_dtype():
    """numpy dtype matching coral_strsv_problem_t (48 bytes)."""
    import numpy as np
    return np.dtype([("uplo", "<i4"), ("trans", "<i4"), ("diag", "<i4"), ("n", "<i4"),
                     ("a", "<u8"), ("x", "<u8"), ("lda", "<i8"), ("incx", "<i8")])


def sgemm_grouped(input_type, count, problems) -> None:
    """Grouped SGEMM over `count` descriptors held in the CUDA tensor `problems`
    (uint8 storage of coral_sgemm_problem_t records)."""
    handle().call("coral_sgemm_grouped", int(input_type), count, C.c_void_p(problems.data_ptr()))


def strsv_batched(count, problems) -> None:
    """Batched STRSV over `count` descriptors held in the CUDA tensor `problems`."""
    handle().call("coral_strsv_batched", count, C.c_void_p(problems.data_ptr()))


def set_grouped_config(tile_n=None) -> None:
    """N tile widths of the tensor-core grouped GEMM for the instance classes
    n <= 64, <= 128, <= 256, > 256 (None restores the default)."""
    if tile_n is None:
        handle().call("coral_set_grouped_config", None)
    else:
        arr = (C.c_int * 4)(*[int(t) for t in tile_n])
        handle().call("coral_set_grouped_config", arr)


def grouped_config() -> list:
    arr = (C.c_int * 4)()
    handle().call("coral_get_grouped_config", arr)
    return list(arr)


def autotune_sgemm_grouped(input_type, count, problems, reps=3):
    """Exhaustive tuning of the grouped policy on one batch; returns
    (ms per candidate [36], best index, tile widths) and installs the best."""
    ms = (C.c_float * 36)()
    best = C.c_int()
    tn = (C.c_int * 4)()
    handle().call("coral_autotune_sgemm_grouped", int(input_type), count,
                  C.c_void_p(problems.data_ptr()), int(reps), ms, C.byref(best), tn)
    return list(ms), best.value, list(tn)
