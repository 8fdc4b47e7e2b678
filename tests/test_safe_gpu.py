"""The checked API on a B200 (coral_b200/safe.py and coral_b200/host/
coral_safe.hpp): each coral-safe routine through views with offsets and
strides, against the oracle.  Bit-exact where the underlying entry point is
(isamax, saxpy, scopy, sswap, sscal, sger, srot, srotm, srotg, srotmg); the
reference tests' fp32 tolerances elsewhere (sdot 4e-6, the rest 1e-5 of the
summed magnitudes)."""
import os
import subprocess

import numpy as np
import pytest
import torch

from coral_b200 import safe
from coral_b200.safe import MatrixMut, MatrixRef, VectorMut, VectorRef
import oracle

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rnd(n, seed):
    return np.random.default_rng(seed).uniform(-1, 1, n).astype(np.float32)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


N, OX, SX, OY, SY = 1001, 3, 2, 5, 3


def views(seed):
    x = rnd(OX + (N - 1) * SX + 1, seed)
    y = rnd(OY + (N - 1) * SY + 1, seed + 1)
    X, Y = dev(x), dev(y)
    return x, y, X, Y


def test_level1_reductions(cuda):
    x, y, X, Y = views(1)
    xv, yv = x[OX:][::SX][:N], y[OY:][::SY][:N]
    got = safe.sdot(VectorRef.new(X, N, SX, OX), VectorRef.new(Y, N, SY, OY))
    want = oracle.sdot(N, np.ascontiguousarray(xv), 1, np.ascontiguousarray(yv), 1)
    assert abs(got - want) <= 4e-6 * float(np.abs(xv.astype(np.float64) * yv).sum())
    assert abs(safe.sasum(VectorRef.new(X, N, SX, OX)) - float(np.abs(xv.astype(np.float64)).sum())) < 1e-3
    assert abs(safe.snrm2(VectorRef.new(X, N, SX, OX)) - float(np.linalg.norm(xv.astype(np.float64)))) < 1e-4
    assert safe.isamax(VectorRef.new(X, N, SX, OX)) == oracle.isamax(N, np.ascontiguousarray(xv), 1)
    assert safe.sdot(VectorRef.new(X, 0, 0, 0), VectorRef.new(Y, 0, 0, 0)) == 0.0


def test_level1_updates_bit_exact(cuda):
    x, y, X, Y = views(2)
    safe.saxpy(0.37, VectorRef.new(X, N, SX, OX), VectorMut.new(Y, N, SY, OY))
    # strided operands take the two-rounding path of saxpy.rs's strided loop
    want2 = oracle.saxpy(N, np.float32(0.37), x[OX:], SX, y[OY:], SY)
    got = host(Y)
    np.testing.assert_array_equal(got[OY:], want2)
    np.testing.assert_array_equal(got[:OY], y[:OY])
    y = got
    safe.sscal(-1.5, VectorMut.new(X, N, SX, OX))
    gx = host(X)
    np.testing.assert_array_equal(gx[OX:], oracle.sscal(N, np.float32(-1.5), x[OX:], SX))
    x = gx
    safe.srot(VectorMut.new(X, N, SX, OX), VectorMut.new(Y, N, SY, OY), 0.6, 0.8)
    wx, wy = oracle.rot("s", N, x[OX:], SX, y[OY:], SY, np.float32(0.6), np.float32(0.8))
    np.testing.assert_array_equal(host(X)[OX:], wx)
    np.testing.assert_array_equal(host(Y)[OY:], wy)
    x, y = host(X), host(Y)
    p = [-1.0, 1.1, -0.4, 0.7, 0.9]
    safe.srotm(VectorMut.new(X, N, SX, OX), VectorMut.new(Y, N, SY, OY), p)
    wx, wy = oracle.rotm("s", N, x[OX:], SX, y[OY:], SY, p)
    np.testing.assert_array_equal(host(X)[OX:], wx)
    np.testing.assert_array_equal(host(Y)[OY:], wy)
    x, y = host(X), host(Y)
    safe.sswap(VectorMut.new(X, N, SX, OX), VectorMut.new(Y, N, SY, OY))
    wx, wy = oracle.swap(N, x[OX:], SX, y[OY:], SY)
    np.testing.assert_array_equal(host(X)[OX:], wx)
    np.testing.assert_array_equal(host(Y)[OY:], wy)
    x, y = host(X), host(Y)
    safe.scopy(VectorRef.new(X, N, SX, OX), VectorMut.new(Y, N, SY, OY))
    np.testing.assert_array_equal(host(Y)[OY:], oracle.copy(N, x[OX:], SX, y[OY:], SY))


def test_rotation_constructors(cuda):
    r = safe.srotg(3.0, 4.0)
    assert r == tuple(np.float32(v) for v in oracle.rotg("s", 3.0, 4.0))
    d1, d2, x1, p = safe.srotmg(1e-3, 3e2, -4.5, 7.25)
    w = oracle.rotmg("s", np.float32(1e-3), np.float32(3e2), np.float32(-4.5), np.float32(7.25))
    assert (d1, d2, x1) == tuple(np.float32(v) for v in w[:3])
    assert [np.float32(v) for v in p] == [np.float32(v) for v in w[3]]


@pytest.mark.parametrize("op", [0, 1])
def test_sgemv_sger_fused(cuda, op):
    m, n, lda, oa = 300, 211, 305, 7
    a = rnd(oa + (n - 1) * lda + m, 10 + op)
    A = dev(a)
    av = a[oa + np.arange(n)[None, :] * lda + np.arange(m)[:, None]].astype(np.float64)   # logical m x n
    xl, yl = (n, m) if op == 0 else (m, n)
    x = rnd(2 + (xl - 1) * 3 + 1, 20 + op)
    y = rnd(1 + (yl - 1) * 2 + 1, 30 + op)
    X, Y = dev(x), dev(y)
    xs, ys = x[2:][::3][:xl].astype(np.float64), y[1:][::2][:yl].astype(np.float64)
    opA = av if op == 0 else av.T
    safe.sgemv(safe.CoralTranspose(op), 1.5, 0.5, MatrixRef.new(A, m, n, lda, oa), VectorRef.new(X, xl, 3, 2),
               VectorMut.new(Y, yl, 2, 1))
    got = host(Y)[1:][::2][:yl]
    scale = 1.5 * (np.abs(opA) @ np.abs(xs)) + 0.5 * np.abs(ys)
    assert (np.abs(got - (1.5 * opA @ xs + 0.5 * ys)) <= 1e-5 * scale).all()
    # fused: y += op(A) x with views (strided output for sdotf goes through SGEMV T)
    y2 = host(Y).copy()
    fn = safe.saxpyf if op == 0 else safe.sdotf
    fn(MatrixRef.new(A, m, n, lda, oa), VectorRef.new(X, xl, 3, 2), VectorMut.new(Y, yl, 2, 1))
    ys2 = y2[1:][::2][:yl].astype(np.float64)
    got = host(Y)[1:][::2][:yl]
    assert (np.abs(got - (opA @ xs + ys2)) <= 1e-5 * (np.abs(opA) @ np.abs(xs) + np.abs(ys2))).all()
    if op == 1:   # contiguous sdotf output through coral_sdotf
        z = rnd(n, 40)
        Z = dev(z)
        safe.sdotf(MatrixRef.new(A, m, n, lda, oa), VectorRef.new(X, m, 3, 2), VectorMut.new(Z, n, 1, 0))
        assert (np.abs(host(Z) - (av.T @ xs + z)) <= 1e-5 * (np.abs(av.T) @ np.abs(xs) + np.abs(z))).all()
    # sger on the same matrix: bit-exact against the strided oracle restatement
    u = rnd(m, 50)
    v = rnd(n, 51)
    safe.sger(0.25, MatrixMut.new(A, m, n, lda, oa), VectorRef.new(dev(u), m, 1, 0), VectorRef.new(dev(v), n, 1, 0))
    want = oracle.sger(m, n, np.float32(0.25), u, 1, v, 1, np.ascontiguousarray(a[oa:]), lda)
    np.testing.assert_array_equal(host(A)[oa:], want)
    np.testing.assert_array_equal(host(A)[:oa], a[:oa])


def test_strsv_view(cuda):
    n, lda, off = 300, 302, 11
    a = rnd(off + (n - 1) * lda + n, 60)
    a[off + np.arange(n) * lda + np.arange(n)] = n
    b = rnd(4 + (n - 1) * 2 + 1, 61)
    B = dev(b)
    safe.strsv(safe.CoralTriangular.Lower, safe.CoralTranspose.NoTrans, safe.CoralDiagonal.NonUnit,
               MatrixRef.new(dev(a), n, n, lda, off), VectorMut.new(B, n, 2, 4))
    xs = host(B)[4:][::2][:n].astype(np.float64)
    Ld = np.tril(a[off + np.arange(n)[None, :] * lda + np.arange(n)[:, None]].astype(np.float64))
    assert np.abs(Ld @ xs - b[4:][::2][:n]).max() < 1e-4


def test_cpp_api(cuda, tmp_path):
    exe = tmp_path / "safe_api_test"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "coral_b200", "host"),
                    "-I", "/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "safe_api_test.cpp"),
                    "-o", str(exe), "-L", os.path.join(ROOT, "coral_b200"), "-lcoral_b200",
                    "-L", "/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath," + os.path.join(ROOT, "coral_b200")],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
