"""Host-slice entry points: operands in host memory, copies inside the call.

coral_host_sgemm takes a single copy each way for small problems and, from
64 MiB of operands, streams column panels of op(B) and C through separate
copy-in / copy-out streams.  Both paths are checked against a float64 torch
product with the component-wise bound used for the device API
(|C - C_ref| <= tol (|alpha| |op(A)||op(B)| + |beta||C|), tol 1e-5), for all
four transpose pairs with padded leading dimensions, ragged last panels,
pageable and pinned host buffers, and beta == 0 with NaN in C (C is then not
read, as in the reference's f32_edge.rs:37-58).
"""
import ctypes

import numpy as np
import pytest
import torch

import coral_b200 as cb
from coral_b200 import _lib

pytestmark = pytest.mark.gpu
vp = ctypes.c_void_p


def host_sgemm(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    lib = _lib.load()
    ptr = (lambda t: vp(t.data_ptr())) if isinstance(a, torch.Tensor) else (lambda t: vp(t.ctypes.data))
    st = lib.coral_host_sgemm(op_a, op_b, m, n, k, alpha, ptr(a), lda, ptr(b), ldb, beta, ptr(c), ldc)
    assert st == 0, st


def check(op_a, op_b, m, n, k, lda, ldb, ldc, alpha, beta, seed, pinned=False, nan_c=False):
    rng = np.random.default_rng(seed)
    ar, ac = (m, k) if op_a == 0 else (k, m)
    br, bc = (k, n) if op_b == 0 else (n, k)
    a = rng.uniform(-1, 1, (ac, lda)).astype(np.float32)   # [col][row]
    b = rng.uniform(-1, 1, (bc, ldb)).astype(np.float32)
    c = rng.uniform(-1, 1, (n, ldc)).astype(np.float32)
    if nan_c:
        c[:, :m] = np.nan
    c0 = c.copy()
    A = torch.from_numpy(a[:, :ar]).double().cuda().T       # stored rows x cols
    B = torch.from_numpy(b[:, :br]).double().cuda().T
    opA = A if op_a == 0 else A.T
    opB = B if op_b == 0 else B.T
    C0 = torch.from_numpy(c0[:, :m]).double().cuda().T
    want = alpha * (opA @ opB)
    mag = abs(alpha) * (opA.abs() @ opB.abs())
    if beta != 0:
        want = want + beta * C0
        mag = mag + abs(beta) * C0.abs()
    if pinned:
        at, bt, ct = (torch.from_numpy(x).pin_memory() for x in (a, b, c))
        host_sgemm(op_a, op_b, m, n, k, alpha, at, lda, bt, ldb, beta, ct, ldc)
        c = ct.numpy()
    else:
        host_sgemm(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    got = torch.from_numpy(c[:, :m]).double().cuda().T
    assert torch.isfinite(got).all()
    assert ((got - want).abs() <= 1e-5 * mag + 1e-6).all()
    np.testing.assert_array_equal(c[:, m:], c0[:, m:])    # rows past m untouched


@pytest.fixture(params=[0, 1], ids=["native", "split_bf16x3"])
def host_mode(request, cuda):
    lib = _lib.load()
    assert lib.coral_host_set_gemm_mode(request.param) == 0
    yield request.param
    lib.coral_host_set_gemm_mode(0)


@pytest.mark.parametrize("op_a,op_b", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_host_sgemm_single_copy(host_mode, op_a, op_b):
    check(op_a, op_b, 300, 200, 100, 305, 310, 303, 1.5, 0.5, 1)


@pytest.mark.parametrize("op_a,op_b", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_host_sgemm_pipelined(host_mode, op_a, op_b):
    # 4096 x 2600 x 2048: > 64 MiB of operands, 6 panels of 512 + one of 40
    m, n, k = 4096, 2600, 2048
    lda = (m if op_a == 0 else k) + 4
    ldb = (k if op_b == 0 else n) + 8
    check(op_a, op_b, m, n, k, lda, ldb, m + 4, 0.75, -1.25, 2)


def test_host_sgemm_pipelined_pinned_beta0_nan(host_mode):
    check(0, 0, 4096, 4096, 1024, 4096, 1024, 4096, 2.0, 0.0, 3, pinned=True, nan_c=True)


def test_host_sgemm_bad_args_before_copies(cuda):
    lib = _lib.load()
    a = np.zeros(16, np.float32)
    st = lib.coral_host_sgemm(0, 0, 4, 4, 4, 1.0, vp(a.ctypes.data), 2, vp(a.ctypes.data), 4, 0.0,
                              vp(a.ctypes.data), 4)
    assert st == 1  # CORAL_ERR_INVALID_ARG (lda < m)
