"""Grouped SGEMM and batched STRSV (no reference counterpart; each instance
has coral_sgemm / coral_strsv semantics) against the oracle.

GEMM: component-wise tolerance 1e-5 (fp32 accumulation, k <= 512); bf16
inputs are compared with the oracle on the bf16-rounded operands.  TRSV:
1e-4, the reference's STRSV tolerance (strsv_tests.rs:213-214).  The grouped
GEMM is also replayed inside a captured CUDA graph.
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle

pytestmark = pytest.mark.gpu


def log_uniform(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size)).astype(np.int64)


def make_gemm_batch(count, lo, hi, seed, bf16=False):
    rng = np.random.default_rng(seed)
    dims = log_uniform(rng, lo, hi, (count, 3))
    ops = np.where(rng.uniform(size=count) < 0.5, 0, 1)   # 50% NN / 50% TN
    host, tensors = [], []
    rec = np.zeros(count, dtype=cb.sgemm_problem_dtype())
    for i in range(count):
        m, n, k = (int(v) for v in dims[i])
        op_a = int(ops[i])
        lda = (m if op_a == 0 else k) + int(rng.integers(0, 3))
        ldb = k + int(rng.integers(0, 3))
        ldc = m + int(rng.integers(0, 3))
        a = rng.uniform(-1, 1, lda * (k if op_a == 0 else m)).astype(np.float32)
        b = rng.uniform(-1, 1, ldb * n).astype(np.float32)
        c = rng.uniform(-1, 1, ldc * n).astype(np.float32)
        if bf16:
            A = torch.from_numpy(a).cuda().to(torch.bfloat16)
            B = torch.from_numpy(b).cuda().to(torch.bfloat16)
            a = A.float().cpu().numpy()
            b = B.float().cpu().numpy()
        else:
            A, B = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        Cd = torch.from_numpy(c).cuda()
        alpha, beta = [(1.5, 0.5), (1.0, 0.0), (-0.5, 1.0), (0.0, 0.7)][i % 4]
        rec[i] = (op_a, 0, m, n, k, alpha, beta, 0, A.data_ptr(), B.data_ptr(), Cd.data_ptr(), lda, ldb, ldc)
        host.append((op_a, m, n, k, alpha, beta, a, lda, b, ldb, c, ldc))
        tensors += [A, B, Cd]
    desc = torch.from_numpy(rec.view(np.uint8)).cuda()
    return host, tensors, desc


def check_gemm_batch(host, tensors, tol, samples=None, seed=0):
    rng = np.random.default_rng(seed)
    torch.cuda.synchronize()
    for i, (op_a, m, n, k, alpha, beta, a, lda, b, ldb, c, ldc) in enumerate(host):
        got = tensors[3 * i + 2].cpu().numpy().reshape(n, ldc).T
        if samples is None:
            ii, jj = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
            ii, jj = ii.ravel(), jj.ravel()
        else:
            ii, jj = rng.integers(0, m, samples), rng.integers(0, n, samples)
        want, bound = oracle.gemm_sample(op_a, 0, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ii, jj)
        err = np.abs(got[ii, jj] - want)
        assert (err <= tol * bound + 1e-30).all(), (i, m, n, k, float((err / np.maximum(bound, 1e-30)).max()))
        np.testing.assert_array_equal(got[m:, :], c.reshape(n, ldc).T[m:, :])


@pytest.mark.parametrize("bf16", [False, True])
def test_grouped_sgemm_small_full_check(cuda, bf16):
    host, tensors, desc = make_gemm_batch(150, 1, 160, seed=3, bf16=bf16)
    cb.sgemm_grouped(1 if bf16 else 0, len(host), desc)
    check_gemm_batch(host, tensors, 1e-5)


def test_grouped_sgemm_4096_instances_graph(cuda):
    """The batched configuration: 4096 instances, m, n, k log-uniform in
    [16, 512], 50% NN / 50% TN, one captured-graph replay."""
    host, tensors, desc = make_gemm_batch(4096, 16, 512, seed=5)
    cb.sgemm_grouped(0, len(host), desc)          # sizes the scratch, outside capture
    torch.cuda.synchronize()
    # restore C, then replay the same work through a CUDA graph
    for i, h in enumerate(host):
        tensors[3 * i + 2].copy_(torch.from_numpy(h[10]))
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            cb.sgemm_grouped(0, len(host), desc)
    torch.cuda.current_stream().wait_stream(s)
    g.replay()
    check_gemm_batch(host, tensors, 1e-5, samples=8)


def test_strsv_batched(cuda):
    rng = np.random.default_rng(8)
    count = 96
    ns = log_uniform(rng, 32, 1024, count)
    rec = np.zeros(count, dtype=cb.strsv_problem_dtype())
    host, keep = [], []
    for i in range(count):
        n = int(ns[i])
        uplo, trans, diag = int(i % 2), int((i // 2) % 2), int((i // 4) % 2)
        lda = n + int(rng.integers(0, 4))
        a = rng.uniform(-1, 1, lda * n).astype(np.float32)
        d = np.arange(n)
        a.reshape(n, lda)[d, d] = np.float32(n) + rng.uniform(0, 1, n).astype(np.float32)
        if diag == 0:
            a = a / np.float32(n)
        incx = 1 if i % 3 else 2
        x = rng.uniform(-1, 1, (n - 1) * incx + 1).astype(np.float32)
        A, X = torch.from_numpy(a).cuda(), torch.from_numpy(x).cuda()
        rec[i] = (uplo, trans, diag, n, A.data_ptr(), X.data_ptr(), lda, incx)
        host.append((uplo, trans, diag, n, a, lda, x, incx))
        keep += [A, X]
    desc = torch.from_numpy(rec.view(np.uint8)).cuda()
    cb.strsv_batched(count, desc)
    torch.cuda.synchronize()
    for i, (uplo, trans, diag, n, a, lda, x, incx) in enumerate(host):
        got = keep[2 * i + 1].cpu().numpy()[::incx][:n]
        want = oracle.strsv(uplo, trans, diag, n, a, lda, x, incx)
        err = np.abs(got - want)
        tol = 1e-4 * np.maximum(np.abs(got), np.abs(want)) + 1e-6
        assert (err <= tol).all(), (i, n, uplo, trans, diag, float(err.max()))
