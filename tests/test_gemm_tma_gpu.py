"""Native SGEMM / DGEMM on TMA-staged tiles (gemm_tma_fma.cu).

The TMA-fed kernel runs when both operands are 16-byte aligned with leading
dimensions that are multiples of 16 bytes; other layouts take the
register-staged kernel.  Both accumulate every output in increasing k with
one fused multiply-add per term, so with alpha = 1 and beta = 0 (no epilogue
arithmetic) the same product computed through the two paths (an aligned
operand, and the same operand shifted one element off the 16-byte boundary)
must agree bit for bit.  Each
result is also checked against the double-double oracle (component-wise
1e-5 for fp32, 1e-13 for fp64) with ragged M, N and K edges, all operation
pairs, and alpha / beta cases of the reference (f32_edge.rs:37-58).
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1, 1), (5, 7, 3), (128, 128, 32), (129, 127, 33), (300, 77, 513), (64, 200, 1000),
          (1000, 1000, 1000)]
OPS = [(0, 0), (0, 1), (1, 0), (1, 1), (2, 2)]


def run_case(dtype, op_a, op_b, m, n, k, alpha, beta, seed):
    es = np.dtype(dtype).itemsize
    q = 16 // es
    rng = np.random.default_rng(seed)
    ar, br = (m if op_a == 0 else k), (k if op_b == 0 else n)
    lda = -(-(ar + 1) // q) * q          # padded to a multiple of 16 bytes
    ldb = -(-(br + 2) // q) * q
    ldc = m + 3
    a = rng.uniform(-1, 1, lda * (k if op_a == 0 else m)).astype(dtype)
    b = rng.uniform(-1, 1, ldb * (n if op_b == 0 else k)).astype(dtype)
    c = rng.uniform(-1, 1, ldc * n).astype(dtype)
    fn = cb.sgemm if dtype == np.float32 else cb.dgemm
    outs = []
    for shift in (0, 1):   # 0: TMA-fed kernel; 1: operands off the 16-byte boundary
        A = torch.from_numpy(np.concatenate([np.zeros(shift, dtype), a])).cuda()[shift:]
        B = torch.from_numpy(np.concatenate([np.zeros(shift, dtype), b])).cuda()[shift:]
        C = torch.from_numpy(c).cuda()
        fn(op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
        torch.cuda.synchronize()
        outs.append(C.cpu().numpy())
    if (alpha, beta) == (1.0, 0.0):   # no epilogue arithmetic: the sums themselves
        np.testing.assert_array_equal(outs[0], outs[1])
    got = outs[0].reshape(n, ldc).T
    sample = 4096 if m * n > 200000 else None
    if sample is None:
        ii, jj = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
        ii, jj = ii.ravel(), jj.ravel()
    else:
        ii, jj = rng.integers(0, m, sample), rng.integers(0, n, sample)
    want, bound = oracle.gemm_sample(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ii, jj)
    tol = 1e-5 if dtype == np.float32 else 1e-13
    err = np.abs(got[ii, jj] - want) / np.maximum(bound, 1e-300)
    assert err.max() <= tol, float(err.max())
    np.testing.assert_array_equal(got[m:, :], c.reshape(n, ldc).T[m:, :])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("ops", OPS)
def test_gemm_tma_vs_register_staged_and_oracle(cuda, dtype, shape, ops):
    m, n, k = shape
    for ci, (alpha, beta) in enumerate([(1.5, 0.5), (1.0, 0.0), (-0.3, 1.0)]):
        run_case(dtype, *ops, m, n, k, alpha, beta, seed=ci + m + n)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_gemm_tma_beta0_ignores_nan_in_c(cuda, dtype):
    m = n = k = 256
    rng = np.random.default_rng(4)
    a = rng.uniform(-1, 1, m * k).astype(dtype)
    b = rng.uniform(-1, 1, k * n).astype(dtype)
    C = torch.full((m * n,), float("nan"), dtype=torch.float32 if dtype == np.float32 else torch.float64,
                   device="cuda")
    fn = cb.sgemm if dtype == np.float32 else cb.dgemm
    fn(0, 0, m, n, k, 2.0, torch.from_numpy(a).cuda(), m, torch.from_numpy(b).cuda(), k, 0.0, C, m)
    torch.cuda.synchronize()
    assert torch.isfinite(C).all()
