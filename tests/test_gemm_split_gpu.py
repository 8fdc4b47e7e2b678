"""Split-BF16 emulated SGEMM/CGEMM on tcgen05 against the double-double oracle.

Component-wise error |C - C_oracle| / (|alpha| |op(A)||op(B)| + |beta||C|):
  SPLIT_BF16X3 (2 pieces, 3 products): dropped terms <= 3 * 2^-18 per product
    in the worst case, random in sign, plus fp32 accumulation -> tol 4e-5
    for small k; the headline 8192^3 case must meet 1e-6.
  SPLIT_BF16X6 (3 pieces, 6 products): fp32-accumulation limited -> tol 1e-5.
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle
from test_gemm_gpu import gemm_case

pytestmark = pytest.mark.gpu

MODES = [(cb.GemmMode.SPLIT_BF16X3, 4e-5), (cb.GemmMode.SPLIT_BF16X6, 1e-5)]


@pytest.fixture(autouse=True)
def restore_mode():
    yield
    cb.set_gemm_mode(cb.GemmMode.NATIVE)


@pytest.mark.parametrize("mode,tol", MODES)
def test_split_smallest(cuda, mode, tol):
    cb.set_gemm_mode(mode)
    gemm_case(cb.sgemm, np.float32, 0, 0, 128, 256, 64, 1.0, 0.0, tol, pad=0)


SHAPES = [(1, 1, 1), (5, 7, 4), (128, 256, 64), (127, 129, 65), (256, 512, 200), (300, 77, 513),
          (1000, 1000, 1000)]


@pytest.mark.parametrize("mode,tol", MODES)
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("ops", [(0, 0), (0, 1), (1, 0), (1, 1), (2, 2)])
def test_sgemm_split_random(cuda, mode, tol, shape, ops):
    cb.set_gemm_mode(mode)
    m, n, k = shape
    sample = 4096 if m * n > 100000 else None
    for alpha, beta in [(1.5, 0.5), (1.0, 0.0), (-0.3, 1.0)]:
        gemm_case(cb.sgemm, np.float32, *ops, m, n, k, alpha, beta, tol, sample=sample)


# Shapes whose dimensions share a residue mod 4, with the pad that makes every
# leading dimension a multiple of 4: the split pre-pass then takes its
# 16-byte kernels (k_split_rows / k_split_cols) with ragged M/N and K edges
# (K not a multiple of 8, M/N not multiples of 4 or 64).
ALIGNED_RAGGED = [((127, 131, 63), 1), ((301, 77, 513), 3), ((66, 70, 10), 2), ((1000, 8, 12), 4)]


@pytest.mark.parametrize("mode,tol", MODES)
@pytest.mark.parametrize("shape,pad", ALIGNED_RAGGED)
@pytest.mark.parametrize("ops", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_sgemm_split_vector_prepass_edges(cuda, mode, tol, shape, pad, ops):
    cb.set_gemm_mode(mode)
    m, n, k = shape
    assert all((d + pad) % 4 == 0 for d in shape)
    gemm_case(cb.sgemm, np.float32, *ops, m, n, k, 1.25, 0.5, tol, pad=pad)


@pytest.mark.parametrize("mode,tol", MODES)
@pytest.mark.parametrize("shape", [(1, 1, 1), (5, 7, 4), (127, 129, 65), (64, 200, 301)])
@pytest.mark.parametrize("ops", [(a, b) for a in (0, 1, 2) for b in (0, 1, 2)])
def test_cgemm_split_random(cuda, mode, tol, shape, ops):
    cb.set_gemm_mode(mode)
    m, n, k = shape
    gemm_case(cb.cgemm, np.complex64, *ops, m, n, k, 1.5 - 0.5j, 0.25 + 1j, 2 * tol)
    gemm_case(cb.cgemm, np.complex64, *ops, m, n, k, 1.0, 0.0, 2 * tol)


def test_cgemm_doctest_split(cuda):
    import fixtures as fx
    d = fx.CGEMM_DOCTEST
    for mode, _ in MODES:
        cb.set_gemm_mode(mode)
        C = torch.from_numpy(d["c"]).cuda()
        cb.cgemm(0, 0, 2, 2, 2, d["alpha"], torch.from_numpy(d["a"]).cuda(), 2,
                 torch.from_numpy(d["b"]).cuda(), 2, d["beta"], C, 2)
        np.testing.assert_array_equal(C.cpu().numpy(), d["expect"])


def _headline(mode, ill_scaled, ops=(0, 0)):
    m = n = k = 8192
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    A = torch.empty(m * k, device="cuda").uniform_(-1, 1, generator=g)
    if ill_scaled:  # rows of A scaled by exp(N(0, 4))
        s = torch.exp(2.0 * torch.randn(m, device="cuda", generator=g))
        A = (A.view(k, m) * s[None, :]).reshape(-1).contiguous()
    B = torch.empty(k * n, device="cuda").uniform_(-1, 1, generator=g)
    C0 = torch.empty(m * n, device="cuda").uniform_(-1, 1, generator=g)
    C = C0.clone()
    cb.set_gemm_mode(mode)
    cb.sgemm(ops[0], ops[1], m, n, k, 1.5, A, m, B, k, 0.5, C, m)
    torch.cuda.synchronize()
    rng = np.random.default_rng(3)
    ii, jj = rng.integers(0, m, 2048), rng.integers(0, n, 2048)
    want, bound = oracle.gemm_sample(ops[0], ops[1], m, n, k, 1.5, A.cpu().numpy(), m,
                                     B.cpu().numpy(), k, 0.5, C0.cpu().numpy(), m, ii, jj)
    got = C.cpu().numpy()[ii + jj * m].astype(np.float64)
    return float((np.abs(got - want) / bound).max())


@pytest.mark.parametrize("ill", [False, True])
def test_sgemm_bf16x3_8192_meets_1e6(cuda, ill):
    err = _headline(cb.GemmMode.SPLIT_BF16X3, ill)
    assert err <= 1e-6, err


def test_sgemm_bf16x3_8192_tt(cuda):
    assert _headline(cb.GemmMode.SPLIT_BF16X3, False, ops=(1, 1)) <= 1e-6


@pytest.mark.parametrize("mode,tol", MODES)
@pytest.mark.parametrize("shape", [(1, 1, 1), (5, 7, 4), (127, 129, 65), (64, 200, 301), (300, 260, 700)])
@pytest.mark.parametrize("ops", [(a, b) for a in (0, 1, 2) for b in (0, 1, 2)])
def test_cgemm_split_3m(cuda, mode, tol, shape, ops):
    """3M mapping: Re = T1 - T2, Im = T3 - T1 - T2 from three real split
    GEMMs.  Against the same component-wise bound as 4M, with three times
    the 4M tolerance: the Im error is bounded by
    (|Re A| + |Im A|)(|Re B| + |Im B|) <= 2 |A||B| plus the T1, T2 terms."""
    h = cb.handle()
    cb.set_gemm_mode(mode)
    h.set_complex_mapping(1)
    try:
        m, n, k = shape
        sample = 4096 if m * n > 50000 else None
        gemm_case(cb.cgemm, np.complex64, *ops, m, n, k, 1.5 - 0.5j, 0.25 + 1j, 6 * tol, sample=sample)
        gemm_case(cb.cgemm, np.complex64, *ops, m, n, k, 1.0, 0.0, 6 * tol, sample=sample)
    finally:
        h.set_complex_mapping(0)
