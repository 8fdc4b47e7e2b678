"""Tensor-core grouped SGEMM (bf16 inputs, and fp32 inputs in split-BF16x3
mode) against the double-double oracle.

No reference counterpart: every instance has coral_sgemm's semantics
(sgemm.rs:106-130, quick returns sgemm_nn.rs:29-45, epilogue
f32_edge.rs:37-58).  Component-wise tolerance 4e-5 of
|alpha| |op(A)| |op(B)| + |beta| |C|, the split-GEMM tests' bound; bf16
inputs are compared with the oracle on the bf16 values themselves.  Cases:
all four operation pairs, padded leading dimensions, unaligned operands,
alpha == 0 and k == 0 instances, K deep enough for several TMEM
accumulation chunks, every tile-width policy, per-instance overrides, the
autotuner, and the 4096-instance configuration replayed in a CUDA graph.
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle

pytestmark = pytest.mark.gpu

TOL = 4e-5


def log_uniform(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size)).astype(np.int64)


def make_batch(count, lo, hi, seed, bf16, all_ops=True, deep=(), zero_k=(), unaligned=False,
               reserved=None):
    rng = np.random.default_rng(seed)
    dims = log_uniform(rng, lo, hi, (count, 3))
    host, keep = [], []
    rec = np.zeros(count, dtype=cb.sgemm_problem_dtype())
    dt = torch.bfloat16 if bf16 else torch.float32
    for i in range(count):
        m, n, k = (int(v) for v in dims[i])
        if i in deep:
            k = 2600
        if i in zero_k:
            k = 0
        op_a = int(rng.integers(0, 2)) if all_ops else int(i % 2)
        op_b = int(rng.integers(0, 2)) if all_ops else 0
        lda = max(m if op_a == 0 else k, 1) + int(rng.integers(0, 3))
        ldb = max(k if op_b == 0 else n, 1) + int(rng.integers(0, 3))
        ldc = m + int(rng.integers(0, 3))
        off = 1 if unaligned and i % 3 == 0 else 0
        a = rng.uniform(-1, 1, lda * max(k if op_a == 0 else m, 1) + off).astype(np.float32)
        b = rng.uniform(-1, 1, ldb * max(n if op_b == 0 else k, 1) + off).astype(np.float32)
        c = rng.uniform(-1, 1, ldc * n).astype(np.float32)
        A = torch.from_numpy(a).cuda().to(dt)
        B = torch.from_numpy(b).cuda().to(dt)
        a = A.float().cpu().numpy()[off:]
        b = B.float().cpu().numpy()[off:]
        Cd = torch.from_numpy(c).cuda()
        alpha, beta = [(1.5, 0.5), (1.0, 0.0), (-0.5, 1.0), (0.0, 0.7), (0.75, -2.0)][i % 5]
        res = 0 if reserved is None else reserved[i % len(reserved)]
        es = A.element_size()
        rec[i] = (op_a, op_b, m, n, k, alpha, beta, res, A.data_ptr() + off * es,
                  B.data_ptr() + off * es, Cd.data_ptr(), lda, ldb, ldc)
        host.append((op_a, op_b, m, n, k, alpha, beta, a, lda, b, ldb, c, ldc))
        keep += [A, B, Cd]
    desc = torch.from_numpy(rec.view(np.uint8)).cuda()
    return host, keep, desc


def restore_c(host, keep):
    for i, h in enumerate(host):
        keep[3 * i + 2].copy_(torch.from_numpy(h[11]))


def check(host, keep, samples=None, seed=0):
    rng = np.random.default_rng(seed)
    torch.cuda.synchronize()
    for i, (op_a, op_b, m, n, k, alpha, beta, a, lda, b, ldb, c, ldc) in enumerate(host):
        got = keep[3 * i + 2].cpu().numpy().reshape(n, ldc).T
        if samples is None or m * n <= samples:
            ii, jj = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
            ii, jj = ii.ravel(), jj.ravel()
        else:
            ii, jj = rng.integers(0, m, samples), rng.integers(0, n, samples)
        want, bound = oracle.gemm_sample(op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ii, jj)
        err = np.abs(got[ii, jj] - want)
        ok = err <= TOL * bound + 1e-30
        assert ok.all(), (i, op_a, op_b, m, n, k, alpha, beta, float((err / np.maximum(bound, 1e-30)).max()))
        np.testing.assert_array_equal(got[m:, :], c.reshape(n, ldc).T[m:, :])


def run(bf16, count, desc):
    h = cb.handle()
    h.set_gemm_mode(cb.GemmMode.SPLIT_BF16X3)
    try:
        cb.sgemm_grouped(1 if bf16 else 0, count, desc)
    finally:
        h.set_gemm_mode(cb.GemmMode.NATIVE)


@pytest.mark.parametrize("bf16", [False, True])
def test_grouped_tc_all_ops_full_check(cuda, bf16):
    host, keep, desc = make_batch(160, 1, 300, seed=11 + bf16, bf16=bf16, zero_k=(7, 8))
    run(bf16, len(host), desc)
    check(host, keep)


@pytest.mark.parametrize("bf16", [False, True])
def test_grouped_tc_unaligned_and_deep_k(cuda, bf16):
    """Operands one element past a 16-byte boundary (the scalar load path)
    and instances with k = 2600 (three TMEM accumulation chunks)."""
    host, keep, desc = make_batch(40, 8, 400, seed=21 + bf16, bf16=bf16, deep=(1, 5, 9),
                                  unaligned=True)
    run(bf16, len(host), desc)
    check(host, keep, samples=4096)


@pytest.mark.parametrize("policy", [(64, 64, 64, 64), (128, 128, 128, 128), (64, 128, 256, 256),
                                    (128, 64, 256, 128)])
def test_grouped_tc_policies(cuda, policy):
    host, keep, desc = make_batch(120, 16, 600, seed=31, bf16=True)
    cb.set_grouped_config(policy)
    try:
        assert cb.grouped_config() == list(policy)
        run(True, len(host), desc)
    finally:
        cb.set_grouped_config(None)
    check(host, keep, samples=2048)


def test_grouped_tc_reserved_override(cuda):
    host, keep, desc = make_batch(90, 16, 600, seed=41, bf16=False, reserved=(64, 128, 256, 0))
    run(False, len(host), desc)
    check(host, keep, samples=2048)


def test_grouped_tc_autotune(cuda):
    host, keep, desc = make_batch(300, 16, 512, seed=51, bf16=True, all_ops=False)
    try:
        ms, best, tile_n = cb.autotune_sgemm_grouped(1, len(host), desc, reps=1)
        assert len(ms) == 36 and 0 <= best < 36 and all(v > 0 for v in ms)
        assert ms[best] == min(ms)
        assert cb.grouped_config() == tile_n
        restore_c(host, keep)
        run(True, len(host), desc)
        check(host, keep, samples=1024)
    finally:
        cb.set_grouped_config(None)


@pytest.mark.parametrize("bf16", [False, True])
def test_grouped_tc_4096_instances_graph(cuda, bf16):
    """The batched configuration: 4096 instances, m, n, k log-uniform in
    [16, 512], 50% NN / 50% TN, replayed from a captured CUDA graph."""
    host, keep, desc = make_batch(4096, 16, 512, seed=61 + bf16, bf16=bf16, all_ops=False)
    run(bf16, len(host), desc)  # sizes the scratch outside capture
    torch.cuda.synchronize()
    restore_c(host, keep)
    h = cb.handle()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    h.set_gemm_mode(cb.GemmMode.SPLIT_BF16X3)
    try:
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                cb.sgemm_grouped(1 if bf16 else 0, len(host), desc)
    finally:
        h.set_gemm_mode(cb.GemmMode.NATIVE)
    torch.cuda.current_stream().wait_stream(s)
    g.replay()
    check(host, keep, samples=16)
    del g
    h.sync()
