"""Checked views and routines over device buffers, after coral-safe.

coral-safe (coral-safe/src/types.rs, errors.rs) validates every vector and
matrix once, when its view is built, and its routines then take views
instead of (slice, n, inc) triples.  This module keeps that API over the
B200 engine's C ABI:

- ``VectorRef`` / ``VectorMut`` (data, n, stride, offset) and ``MatrixRef``
  / ``MatrixMut`` (data, n_rows, n_cols, lda, offset) are built with
  ``new(...)``, which raises :class:`BufferError` with the reference's variant
  and fields (types.rs:76-103, 174-201).  ``data`` is a 1-D torch tensor, and
  lengths count its elements.
- The routines (level 1, ``sgemv``, ``sger``, ``strsv``, fused ``saxpyf`` /
  ``sdotf``) take views and call the ``coral_*`` entry points at
  ``data_ptr() + offset``.  The data must then live on the GPU.  Logical
  lengths that disagree raise ``ValueError``; the reference checks them with
  ``debug_assert!`` (types.rs:324-332, sgemv_n.rs:23-24, sger.rs:227-228).

Empty views (n == 0, or a matrix with no rows or columns) skip every check,
as in the reference, and the routines return at once on them.
"""
from __future__ import annotations

import ctypes as C
import enum

from .blas import CoralError, handle  # noqa: F401  (CoralError re-exported for callers)

_USIZE_MAX = (1 << 64) - 1


class CoralTranspose(enum.IntEnum):
    """coral-safe/src/types.rs: NoTrans, Trans."""
    NoTrans = 0
    Trans = 1


class CoralTriangular(enum.IntEnum):
    Upper = 0
    Lower = 1


class CoralDiagonal(enum.IntEnum):
    Unit = 0
    NonUnit = 1

    def is_unit(self) -> bool:
        return self is CoralDiagonal.Unit


class BufferError(Exception):
    """errors.rs: ZeroStride, OutOfBounds{required, len}, BadOffset{offset,
    len}, InvalidLda{lda, n_rows}, with the reference's Display text."""

    def __init__(self, kind: str, **fields):
        self.kind = kind
        self.fields = fields
        super().__init__(self._text())

    def _text(self) -> str:
        f = self.fields
        if self.kind == "ZeroStride":
            return "stride must be nonzero"
        if self.kind == "OutOfBounds":
            return f"buffer too small: required {f['required']}, have {f['len']}"
        if self.kind == "BadOffset":
            return f"offset {f['offset']} out of range for buffer of len {f['len']}"
        return f"leading dimension {f['lda']} must exceed num rows {f['n_rows']}"

    def __eq__(self, other) -> bool:
        return isinstance(other, BufferError) and (self.kind, self.fields) == (other.kind, other.fields)

    def __hash__(self):
        return hash((self.kind, tuple(sorted(self.fields.items()))))

    @classmethod
    def ZeroStride(cls):
        return cls("ZeroStride")

    @classmethod
    def OutOfBounds(cls, required: int, len: int):  # noqa: A002 (the reference's field name)
        return cls("OutOfBounds", required=required, len=len)

    @classmethod
    def BadOffset(cls, offset: int, len: int):  # noqa: A002
        return cls("BadOffset", offset=offset, len=len)

    @classmethod
    def InvalidLda(cls, lda: int, n_rows: int):
        return cls("InvalidLda", lda=lda, n_rows=n_rows)


def _len(data) -> int:
    if data.dim() != 1:
        raise TypeError("view data must be a 1-D tensor")
    return int(data.numel())


def _sat(v: int) -> int:
    """usize saturating arithmetic of the reference's length checks."""
    return min(v, _USIZE_MAX)


class _Vector:
    def __init__(self, data, n, stride, offset):
        self._data, self._n, self._stride, self._offset = data, n, stride, offset

    @classmethod
    def new(cls, data, n: int, stride: int, offset: int):
        """types.rs:76-103: n == 0 skips the checks; stride 0 -> ZeroStride;
        (n - 1) stride + offset + 1 elements must fit -> OutOfBounds."""
        length = _len(data)
        if n == 0:
            return cls(data, n, stride, offset)
        if stride == 0:
            raise BufferError.ZeroStride()
        required = _sat(_sat(_sat((n - 1) * stride) + offset) + 1)
        if required > length:
            raise BufferError.OutOfBounds(required, length)
        return cls(data, n, stride, offset)

    def n(self) -> int:
        return self._n

    def stride(self) -> int:
        return self._stride

    def offset(self) -> int:
        return self._offset

    def as_slice(self):
        return self._data

    def contiguous_slice(self):
        return self._data[self._offset:self._offset + self._n] if self._stride == 1 else None

    def compare_n(self, n: int) -> bool:
        return self._n == n

    def _ptr(self):
        return C.c_void_p(self._data.data_ptr() + self._offset * self._data.element_size())


class VectorRef(_Vector):
    """A read-only strided vector view (types.rs: VectorRef)."""


class VectorMut(_Vector):
    """A writable strided vector view (types.rs: VectorMut)."""

    def as_slice_mut(self):
        return self._data

    def contiguous_slice_mut(self):
        return self.contiguous_slice()


class _Matrix:
    def __init__(self, data, n_rows, n_cols, lda, offset):
        self._data, self._m, self._n, self._lda, self._offset = data, n_rows, n_cols, lda, offset

    @classmethod
    def new(cls, data, n_rows: int, n_cols: int, lda: int, offset: int):
        """types.rs:174-201: an empty matrix skips the checks; lda 0 ->
        ZeroStride; lda < n_rows -> InvalidLda; (n_cols - 1) lda + n_rows +
        offset elements must fit -> OutOfBounds."""
        length = _len(data)
        if n_rows == 0 or n_cols == 0:
            return cls(data, n_rows, n_cols, lda, offset)
        if lda == 0:
            raise BufferError.ZeroStride()
        if lda < n_rows:
            raise BufferError.InvalidLda(lda, n_rows)
        required = _sat(_sat(_sat((n_cols - 1) * lda) + n_rows) + offset)
        if required > length:
            raise BufferError.OutOfBounds(required, length)
        return cls(data, n_rows, n_cols, lda, offset)

    def n_rows(self) -> int:
        return self._m

    def n_cols(self) -> int:
        return self._n

    def lda(self) -> int:
        return self._lda

    def offset(self) -> int:
        return self._offset

    def as_slice(self):
        return self._data

    def contiguous_slice(self):
        if self._lda != self._m:
            return None
        return self._data[self._offset:self._offset + (self._n - 1) * self._lda + self._m]

    def compare_m_n(self) -> bool:
        return self._m == self._n

    def _ptr(self):
        return C.c_void_p(self._data.data_ptr() + self._offset * self._data.element_size())


class MatrixRef(_Matrix):
    """A read-only column-major matrix view (types.rs: MatrixRef)."""


class MatrixMut(_Matrix):
    """A writable column-major matrix view (types.rs: MatrixMut)."""

    def as_slice_mut(self):
        return self._data

    def contiguous_slice_mut(self):
        return self.contiguous_slice()


# ---- routines ------------------------------------------------------------------
def _empty(v) -> bool:
    return v.n() == 0 if isinstance(v, _Vector) else (v.n_rows() == 0 or v.n_cols() == 0)


def _f32_views(*views):
    """Non-empty views must hold float32 CUDA data (empty ones are never read:
    the entry points return before touching their pointers)."""
    import torch
    for v in views:
        if _empty(v):
            continue
        t = v.as_slice()
        if not t.is_cuda:
            raise TypeError("the view's data must be a CUDA tensor")
        if t.dtype != torch.float32:
            raise TypeError(f"the view's data has dtype {t.dtype}, expected torch.float32")


def _same_n(x, y) -> None:
    """debug_assert_n_eq! (types.rs:324-332)."""
    if not x.compare_n(y.n()):
        raise ValueError("number of logical elements must be equal")


def _scalar(name, *args, ctype=C.c_float):
    r = ctype()
    handle().call(name, *args, C.cast(C.byref(r), C.c_void_p))
    return r.value


def isamax(x: VectorRef) -> int:
    """coral-safe level1/isamax.rs:27: 0-based index of the first max |x_i|."""
    _f32_views(x)
    return _scalar("coral_isamax", x.n(), x._ptr(), x.stride(), ctype=C.c_size_t)


def sasum(x: VectorRef) -> float:
    """level1/sasum.rs:26."""
    _f32_views(x)
    return _scalar("coral_sasum", x.n(), x._ptr(), x.stride())


def snrm2(x: VectorRef) -> float:
    """level1/snrm2.rs:25."""
    _f32_views(x)
    return _scalar("coral_snrm2", x.n(), x._ptr(), x.stride())


def sdot(x: VectorRef, y: VectorRef) -> float:
    """level1/sdot.rs:28."""
    _same_n(x, y)
    _f32_views(x, y)
    return _scalar("coral_sdot", x.n(), x._ptr(), x.stride(), y._ptr(), y.stride())


def saxpy(alpha: float, x: VectorRef, y: VectorMut) -> None:
    """level1/saxpy.rs:27."""
    _same_n(x, y)
    _f32_views(x, y)
    handle().call("coral_saxpy", x.n(), C.c_float(alpha), x._ptr(), x.stride(), y._ptr(), y.stride())


def scopy(x: VectorRef, y: VectorMut) -> None:
    """level1/scopy.rs:26."""
    _same_n(x, y)
    _f32_views(x, y)
    handle().call("coral_scopy", x.n(), x._ptr(), x.stride(), y._ptr(), y.stride())


def sswap(x: VectorMut, y: VectorMut) -> None:
    """level1/sswap.rs:24."""
    _same_n(x, y)
    _f32_views(x, y)
    handle().call("coral_sswap", x.n(), x._ptr(), x.stride(), y._ptr(), y.stride())


def sscal(alpha: float, x: VectorMut) -> None:
    """level1/sscal.rs:25."""
    _f32_views(x)
    handle().call("coral_sscal", x.n(), C.c_float(alpha), x._ptr(), x.stride())


def srot(x: VectorMut, y: VectorMut, c: float, s: float) -> None:
    """level1/srot.rs:32."""
    _same_n(x, y)
    _f32_views(x, y)
    handle().call("coral_srot", x.n(), x._ptr(), x.stride(), y._ptr(), y.stride(), C.c_float(c), C.c_float(s))


def srotm(x: VectorMut, y: VectorMut, param) -> None:
    """level1/srotm.rs:94: param = [flag, h11, h21, h12, h22]."""
    _same_n(x, y)
    _f32_views(x, y)
    p = (C.c_float * 5)(*[float(v) for v in param])
    handle().call("coral_srotm", x.n(), x._ptr(), x.stride(), y._ptr(), y.stride(), C.cast(p, C.c_void_p))


def srotg(a: float, b: float):
    """level1/srotg.rs:34: returns the updated (a, b) and (c, s) as (r, z, c, s)."""
    v = [C.c_float(a), C.c_float(b), C.c_float(), C.c_float()]
    handle().call("coral_srotg", *[C.cast(C.byref(t), C.c_void_p) for t in v])
    return tuple(t.value for t in v)


def srotmg(sd1: float, sd2: float, sx1: float, sy1: float):
    """level1/srotmg.rs:32: returns (sd1, sd2, sx1, param)."""
    v = [C.c_float(sd1), C.c_float(sd2), C.c_float(sx1)]
    p = (C.c_float * 5)()
    handle().call("coral_srotmg", *[C.cast(C.byref(t), C.c_void_p) for t in v], C.c_float(sy1),
                  C.cast(p, C.c_void_p))
    return v[0].value, v[1].value, v[2].value, list(p)


def sgemv(op: CoralTranspose, alpha: float, beta: float, a: MatrixRef, x: VectorRef, y: VectorMut) -> None:
    """level2/sgemv.rs:29: y <- alpha op(A) x + beta y."""
    m, n = a.n_rows(), a.n_cols()
    xn, yn = (n, m) if op == CoralTranspose.NoTrans else (m, n)
    if not x.compare_n(xn):
        raise ValueError(f"logical length of x must equal {'n_cols' if xn == n else 'n_rows'}")
    if not y.compare_n(yn):
        raise ValueError(f"logical length of y must equal {'n_rows' if yn == m else 'n_cols'}")
    _f32_views(x, y)
    if m == 0 or n == 0:
        return
    _f32_views(a)
    handle().call("coral_sgemv", int(op), m, n, C.c_float(alpha), a._ptr(), a.lda(), x._ptr(), x.stride(),
                  C.c_float(beta), y._ptr(), y.stride())


def sger(alpha: float, a: MatrixMut, x: VectorRef, y: VectorRef) -> None:
    """level2/sger.rs:218: A += alpha x y^T."""
    if y.n() != a.n_cols():
        raise ValueError("logical length of y must equal n_cols")
    if x.n() != a.n_rows():
        raise ValueError("logical length of x must equal n_rows")
    if a.n_rows() == 0 or a.n_cols() == 0:
        return
    _f32_views(a, x, y)
    handle().call("coral_sger", a.n_rows(), a.n_cols(), C.c_float(alpha), x._ptr(), x.stride(), y._ptr(),
                  y.stride(), a._ptr(), a.lda())


def strsv(uplo: CoralTriangular, trans: CoralTranspose, diag: CoralDiagonal, a: MatrixRef, x: VectorMut) -> None:
    """level2/strsv.rs:27: solve op(A) x = b in place, A triangular n x n."""
    if not a.compare_m_n():
        raise ValueError("matrix must be square")
    if not x.compare_n(a.n_rows()):
        raise ValueError("logical length of x must equal n")
    n = a.n_rows()
    if n == 0:
        return
    _f32_views(a, x)
    handle().call("coral_strsv", int(uplo), int(trans), int(diag), n, a._ptr(), a.lda(), x._ptr(), x.stride())


def saxpyf(a: MatrixRef, x: VectorRef, y: VectorMut) -> None:
    """fused/saxpyf.rs:162: y += A x."""
    if not x.compare_n(a.n_cols()):
        raise ValueError("logical length of x must equal n_cols")
    if not y.compare_n(a.n_rows()):
        raise ValueError("logical length of y must equal n_rows")
    if a.n_rows() == 0 or a.n_cols() == 0:
        return
    _f32_views(a, x, y)
    handle().call("coral_saxpyf", a.n_rows(), a.n_cols(), x._ptr(), x.stride(), a._ptr(), a.lda(), y._ptr(),
                  y.stride())


def sdotf(a: MatrixRef, x: VectorRef, y: VectorMut) -> None:
    """fused/sdotf.rs:162: y += A^T x.  coral_sdotf writes a contiguous
    output, as the reference's sdotf does; a strided y goes through SGEMV T
    with alpha = beta = 1, the same sum."""
    if not x.compare_n(a.n_rows()):
        raise ValueError("logical length of x must equal n_rows")
    if not y.compare_n(a.n_cols()):
        raise ValueError("logical length of y must equal n_cols")
    if a.n_rows() == 0 or a.n_cols() == 0:
        return
    _f32_views(a, x, y)
    if y.stride() == 1:
        handle().call("coral_sdotf", a.n_rows(), a.n_cols(), a._ptr(), a.lda(), x._ptr(), x.stride(), y._ptr())
        return
    # strided output: y += A^T x as sgemv T with alpha = beta = 1
    handle().call("coral_sgemv", 1, a.n_rows(), a.n_cols(), C.c_float(1.0), a._ptr(), a.lda(), x._ptr(),
                  x.stride(), C.c_float(1.0), y._ptr(), y.stride())
