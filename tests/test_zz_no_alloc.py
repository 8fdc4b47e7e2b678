"""The allocation-free split-BF16x3 SGEMM entry point, called through the C ABI.

coral_sgemm_bf16x3_noalloc exists for callers that must not have device
memory allocated on their behalf (a process that owns all of HBM through its
own sub-allocator, a latency-critical loop that cannot take cudaMalloc's
implicit synchronisation, a deployment that forbids device allocation after
start-up).  Its operand pieces live in a fixed 32 MiB device array shared by
every call.  This file is collected last on purpose; it must pass alone in a
fresh process as well as after the other tests.

Each result is compared with the existing entry point (coral_sgemm in
CORAL_GEMM_SPLIT_BF16X3 mode) on the same inputs, with the component-wise
tolerance the split-GEMM tests use (4e-5 of |alpha||op(A)||op(B)| +
|beta||C|, from the double-double oracle), over two calls in a row that reuse
the shared array with different shapes and operations.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle
from coral_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 4e-5


def _operands(op_a, op_b, m, n, k, seed):
    rng = np.random.default_rng(seed)
    lda = (m if op_a == 0 else k) + 1
    ldb = (k if op_b == 0 else n) + 2
    ldc = m + 3
    a = rng.uniform(-1, 1, lda * (k if op_a == 0 else m)).astype(np.float32)
    b = rng.uniform(-1, 1, ldb * (n if op_b == 0 else k)).astype(np.float32)
    c = rng.uniform(-1, 1, ldc * n).astype(np.float32)
    return a, lda, b, ldb, c, ldc


def _run_pair(op_a, op_b, m, n, k, alpha, beta, seed):
    a, lda, b, ldb, c, ldc = _operands(op_a, op_b, m, n, k, seed)
    A, B = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    C_new, C_old = torch.from_numpy(c).cuda(), torch.from_numpy(c).cuda()
    lib = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = lib.coral_sgemm_bf16x3_noalloc(stream, op_a, op_b, m, n, k, alpha,
                                        C.c_void_p(A.data_ptr()), lda, C.c_void_p(B.data_ptr()),
                                        ldb, beta, C.c_void_p(C_new.data_ptr()), ldc)
    assert st == 0, st
    cb.set_gemm_mode(cb.GemmMode.SPLIT_BF16X3)
    try:
        cb.sgemm(op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C_old, ldc)
    finally:
        cb.set_gemm_mode(cb.GemmMode.NATIVE)
    torch.cuda.synchronize()
    got_new = C_new.cpu().numpy().reshape(n, ldc).T
    got_old = C_old.cpu().numpy().reshape(n, ldc).T
    ii, jj = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
    want, bound = oracle.gemm_sample(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                                     ii.ravel(), jj.ravel())
    bound = np.maximum(bound.reshape(m, n), 1e-30)
    assert (np.abs(got_new[:m] - got_old[:m]) / bound).max() <= TOL
    assert (np.abs(got_new[:m] - want.reshape(m, n)) / bound).max() <= TOL
    # rows past m inside the leading dimension stay untouched
    np.testing.assert_array_equal(got_new[m:], c.reshape(n, ldc).T[m:])


def test_noalloc_matches_existing_entry_point_twice(cuda):
    _run_pair(0, 0, 300, 520, 257, 1.5, 0.5, seed=1)
    _run_pair(1, 1, 129, 77, 1000, -0.75, 0.0, seed=2)


def _call(lib, m, n, k, alpha, A, B, beta, Cd, stream=None):
    return lib.coral_sgemm_bf16x3_noalloc(stream, 0, 0, m, n, k, alpha, C.c_void_p(A.data_ptr()),
                                          max(m, 1), C.c_void_p(B.data_ptr()), max(k, 1), beta,
                                          C.c_void_p(Cd.data_ptr()), max(m, 1))


@pytest.mark.parametrize("m,n,k", [(300, 200, 0), (4096, 4096, 4096)])
@pytest.mark.parametrize("beta", [0.0, 1.0, -0.5])
def test_noalloc_scale_only(cuda, m, n, k, beta):
    """alpha == 0 or k == 0 only scales C (sgemm_nn.rs:29-45) and uses no
    scratch, so it succeeds even where the pieces would not fit: beta == 0
    writes zeros, beta == 1 leaves C as it was, other beta scale C."""
    lib = _lib.load()
    A = torch.ones(max(m * k, 1), device="cuda")
    B = torch.ones(max(k * n, 1), device="cuda")
    c = np.random.default_rng(3).uniform(-1, 1, m * n).astype(np.float32)
    Cd = torch.from_numpy(c).cuda()
    alpha = 0.0 if k else 2.0
    assert _call(lib, m, n, k, alpha, A, B, beta, Cd) == 0
    torch.cuda.synchronize()
    got = Cd.cpu().numpy()
    want = np.zeros_like(c) if beta == 0.0 else (c if beta == 1.0 else c * np.float32(beta))
    np.testing.assert_array_equal(got, want)


def test_noalloc_empty_and_huge_sizes(cuda):
    """m == 0 returns at once whatever k is; sizes whose byte count would
    wrap 64 bits are rejected by the size check, not let through."""
    lib = _lib.load()
    assert lib.coral_sgemm_bf16x3_noalloc(None, 0, 0, 0, 4096, 1 << 30, 1.0, None, 1, None,
                                          1 << 30, 0.0, None, 1) == 0
    buf = torch.zeros(4, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    big = (1 << 31) - 1
    # m = n = 2^31 - 1, k = 2^31 - 1: 4 (m + n) kp is about 2^66 bytes
    assert lib.coral_sgemm_bf16x3_noalloc(None, 0, 0, big, big, big, 1.0, p, big, p, big, 0.0, p,
                                          big) == 5
    torch.cuda.synchronize()
    assert float(buf.abs().sum()) == 0.0


def test_noalloc_status_reads_clear_after_normal_calls(cuda):
    lib = _lib.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _run_pair(0, 1, 64, 96, 40, 1.0, 1.0, seed=4)
    assert lib.coral_sgemm_bf16x3_noalloc_status(stream) == 0
    assert lib.coral_sgemm_bf16x3_noalloc_status(None) == 0


def test_noalloc_rejects_sizes_beyond_fixed_scratch(cuda):
    lib = _lib.load()
    m = n = k = 4096  # pieces need 4 * 8192 * 4096 bytes = 128 MiB > 32 MiB
    A = torch.ones(m * k, device="cuda")
    B = torch.ones(k * n, device="cuda")
    C0 = torch.zeros(m * n, device="cuda")
    st = lib.coral_sgemm_bf16x3_noalloc(None, 0, 0, m, n, k, 1.0, C.c_void_p(A.data_ptr()), m,
                                        C.c_void_p(B.data_ptr()), k, 0.0,
                                        C.c_void_p(C0.data_ptr()), m)
    torch.cuda.synchronize()
    assert st == 5  # CORAL_ERR_NOT_SUPPORTED, nothing enqueued
    assert float(C0.abs().sum()) == 0.0
