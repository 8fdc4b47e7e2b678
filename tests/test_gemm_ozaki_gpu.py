"""Ozaki INT8-slice DGEMM / ZGEMM on tcgen05 against the double-double oracle.

7 signed 7-bit slices per operand (49 bits of each row-/column-scaled value),
the 28 slice products with p + q <= 8 summed exactly in INT32: component-wise
error |C - C_oracle| / (|alpha| |op(A)||op(B)| + |beta||C|) <= 1e-13 here
(the native FP64 kernel's tolerance), and on the 4096^3 configuration -- also
with rows of A scaled by exp(N(0, 4)) -- <= 4e-15.
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle
from test_gemm_gpu import gemm_case

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def ozaki_mode():
    cb.set_gemm_mode(cb.GemmMode.OZAKI_INT8)
    yield
    cb.set_gemm_mode(cb.GemmMode.NATIVE)


def test_ozaki_smallest(cuda):
    gemm_case(cb.dgemm, np.float64, 0, 0, 128, 64, 64, 1.0, 0.0, 1e-13, pad=0)


SHAPES = [(1, 1, 1), (5, 7, 4), (128, 64, 64), (127, 129, 65), (256, 512, 200), (300, 77, 513),
          (1000, 1000, 1000)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("ops", [(0, 0), (0, 1), (1, 0), (1, 1), (2, 2)])
def test_dgemm_ozaki_random(cuda, shape, ops):
    m, n, k = shape
    sample = 4096 if m * n > 100000 else None
    for alpha, beta in [(1.5, 0.5), (1.0, 0.0), (-0.3, 1.0)]:
        gemm_case(cb.dgemm, np.float64, *ops, m, n, k, alpha, beta, 1e-13, sample=sample)


@pytest.mark.parametrize("shape", [(1, 1, 1), (5, 7, 4), (127, 129, 65), (64, 200, 301)])
@pytest.mark.parametrize("ops", [(a, b) for a in (0, 1, 2) for b in (0, 1, 2)])
def test_zgemm_ozaki_random(cuda, shape, ops):
    m, n, k = shape
    gemm_case(cb.zgemm, np.complex128, *ops, m, n, k, 1.5 - 0.5j, 0.25 + 1j, 1e-13)
    gemm_case(cb.zgemm, np.complex128, *ops, m, n, k, 1.0, 0.0, 1e-13)


def test_dgemm_ozaki_zero_rows_and_columns(cuda):
    m, n, k = 130, 70, 90
    rng = np.random.default_rng(0)
    a = rng.uniform(-1, 1, m * k)
    b = rng.uniform(-1, 1, k * n)
    a.reshape(k, m)[:, 3] = 0.0     # row 3 of A all zero
    b.reshape(n, k)[5, :] = 0.0     # column 5 of B all zero
    c = rng.uniform(-1, 1, m * n)
    C = torch.from_numpy(c).cuda()
    cb.dgemm(0, 0, m, n, k, 2.0, torch.from_numpy(a).cuda(), m, torch.from_numpy(b).cuda(), k, 0.5, C, m)
    got = C.cpu().numpy().reshape(n, m).T
    ii, jj = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
    want, bound = oracle.gemm_sample(0, 0, m, n, k, 2.0, a, m, b, k, 0.5, c, m, ii.ravel(), jj.ravel())
    assert (np.abs(got.ravel() - want) / bound).max() <= 1e-13


def _dgemm_4096(mode, ill):
    m = n = k = 4096
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    A = torch.empty(m * k, dtype=torch.float64, device="cuda").uniform_(-1, 1, generator=g)
    if ill:
        s = torch.exp(2.0 * torch.randn(m, dtype=torch.float64, device="cuda", generator=g))
        A = (A.view(k, m) * s[None, :]).reshape(-1).contiguous()
    B = torch.empty(k * n, dtype=torch.float64, device="cuda").uniform_(-1, 1, generator=g)
    C0 = torch.empty(m * n, dtype=torch.float64, device="cuda").uniform_(-1, 1, generator=g)
    C = C0.clone()
    cb.set_gemm_mode(mode)
    cb.dgemm(0, 0, m, n, k, 1.5, A, m, B, k, 0.5, C, m)
    torch.cuda.synchronize()
    rng = np.random.default_rng(4)
    ii, jj = rng.integers(0, m, 1024), rng.integers(0, n, 1024)
    want, bound = oracle.gemm_sample(0, 0, m, n, k, 1.5, A.cpu().numpy(), m, B.cpu().numpy(), k,
                                     0.5, C0.cpu().numpy(), m, ii, jj)
    got = C.cpu().numpy()[ii + jj * m]
    return float((np.abs(got - want) / bound).max())


@pytest.mark.parametrize("ill", [False, True])
def test_dgemm_ozaki_4096_accuracy(cuda, ill):
    """Measured: ~1e-15 (Ozaki) vs ~2e-16 (native FP64) component-wise."""
    err_oz = _dgemm_4096(cb.GemmMode.OZAKI_INT8, ill)
    err_native = _dgemm_4096(cb.GemmMode.NATIVE, ill)
    assert err_oz <= 4e-15, (err_oz, err_native)


@pytest.mark.parametrize("shape", [(1, 1, 1), (5, 7, 4), (127, 129, 65), (64, 200, 301), (300, 260, 500)])
@pytest.mark.parametrize("ops", [(a, b) for a in (0, 1, 2) for b in (0, 1, 2)])
def test_zgemm_ozaki_3m(cuda, shape, ops):
    """3M mapping: three real Ozaki GEMMs, Re = T1 - T2, Im = T3 - T1 - T2.
    Same component-wise bound as 4M with three times the tolerance (the Im
    error is bounded by (|Re A| + |Im A|)(|Re B| + |Im B|) <= 2 |A||B| plus the
    T1, T2 terms)."""
    h = cb.handle()
    h.set_complex_mapping(1)
    try:
        m, n, k = shape
        sample = 4096 if m * n > 50000 else None
        gemm_case(cb.zgemm, np.complex128, *ops, m, n, k, 1.5 - 0.5j, 0.25 + 1j, 3e-13, sample=sample)
        gemm_case(cb.zgemm, np.complex128, *ops, m, n, k, 1.0, 0.0, 3e-13, sample=sample)
    finally:
        h.set_complex_mapping(0)
