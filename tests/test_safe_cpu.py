"""The checked API's view validation on the host (coral_b200/safe.py and
coral_b200/host/coral_safe.hpp), after coral-safe/tests/types.rs: ZeroStride,
OutOfBounds{required: 6, len: 5}, InvalidLda{lda: 4, n_rows: 5}, plus empty
views, offsets, usize saturation and the Display text of errors.rs.  No GPU:
views are only validated here, never read."""
import os
import subprocess

import pytest
import torch

from coral_b200 import safe
from coral_b200.safe import BufferError, MatrixMut, MatrixRef, VectorMut, VectorRef

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def buf(n):
    return torch.ones(n, dtype=torch.float32)


def err(fn, *a):
    with pytest.raises(BufferError) as e:
        fn(*a)
    return e.value


def test_zero_stride():
    for cls in (VectorRef, VectorMut):
        assert err(cls.new, buf(5), 5, 0, 0) == BufferError.ZeroStride()


def test_within_bounds():
    for cls in (VectorRef, VectorMut):
        assert err(cls.new, buf(5), 3, 2, 1) == BufferError.OutOfBounds(required=6, len=5)
        v = cls.new(buf(6), 3, 2, 1)
        assert (v.n(), v.stride(), v.offset()) == (3, 2, 1) and v.compare_n(3)


def test_valid_lda():
    for cls in (MatrixRef, MatrixMut):
        assert err(cls.new, buf(24), 5, 6, 4, 0) == BufferError.InvalidLda(lda=4, n_rows=5)
        a = cls.new(buf(42), 5, 6, 7, 0)
        assert (a.n_rows(), a.n_cols(), a.lda(), a.offset()) == (5, 6, 7, 0) and not a.compare_m_n()
        assert err(cls.new, buf(42), 5, 6, 7, 3) == BufferError.OutOfBounds(required=43, len=42)
        assert err(cls.new, buf(42), 5, 6, 0, 0) == BufferError.ZeroStride()


def test_empty_views_skip_checks():
    assert VectorRef.new(buf(0), 0, 0, 99).n() == 0
    assert MatrixRef.new(buf(0), 0, 6, 0, 0).n_cols() == 6
    assert MatrixMut.new(buf(0), 5, 0, 1, 0).n_rows() == 5


def test_saturation_and_slices():
    big = (1 << 64) - 1
    assert err(VectorRef.new, buf(10), big, 2, 0) == BufferError.OutOfBounds(required=big, len=10)
    t = torch.arange(20, dtype=torch.float32)
    assert VectorRef.new(t, 4, 1, 3).contiguous_slice().tolist() == [3, 4, 5, 6]
    assert VectorRef.new(t, 4, 2, 3).contiguous_slice() is None
    assert MatrixRef.new(t, 3, 2, 3, 1).contiguous_slice().tolist() == [1, 2, 3, 4, 5, 6]
    assert MatrixRef.new(t, 3, 2, 4, 1).contiguous_slice() is None


def test_display_text():
    assert str(BufferError.ZeroStride()) == "stride must be nonzero"
    assert str(BufferError.OutOfBounds(6, 5)) == "buffer too small: required 6, have 5"
    assert str(BufferError.BadOffset(9, 4)) == "offset 9 out of range for buffer of len 4"
    assert str(BufferError.InvalidLda(4, 5)) == "leading dimension 4 must exceed num rows 5"


def test_routines_refuse_before_any_call():
    x, y = VectorRef.new(buf(5), 5, 1, 0), VectorRef.new(buf(4), 4, 1, 0)
    with pytest.raises(ValueError):
        safe.sdot(x, y)                       # logical lengths differ
    with pytest.raises(TypeError):
        safe.sdot(x, VectorRef.new(buf(5), 5, 1, 0))   # host data
    a = MatrixRef.new(buf(12), 3, 4, 3, 0)
    with pytest.raises(ValueError):
        safe.strsv(safe.CoralTriangular.Lower, safe.CoralTranspose.NoTrans, safe.CoralDiagonal.NonUnit, a,
                   VectorMut.new(buf(3), 3, 1, 0))
    with pytest.raises(ValueError):
        safe.sgemv(safe.CoralTranspose.Trans, 1.0, 0.0, a, VectorRef.new(buf(4), 4, 1, 0),
                   VectorMut.new(buf(4), 4, 1, 0))


def test_cpp_header_views(tmp_path):
    exe = tmp_path / "safe_views_test"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "coral_b200", "host"),
                    os.path.join(ROOT, "tests", "cpp", "safe_views_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
