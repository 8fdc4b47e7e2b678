"""Split-BF16 SGEMM / CGEMM on CTA-pair tiles (tcgen05 cta_group::2) against
the double-double oracle.

The 256 x 256 tile of a cluster of two CTAs must give the same results as the
single-CTA tiles within the same component-wise bounds (the products are the
same exact bf16 products; only which SM holds which rows changes).  Shapes
cover: the odd CTA's half entirely past m (m <= 128), ragged M/N/K edges,
tiles narrower than the raster group, split-K over pair tiles, the complex 4M
mapping and the 3-piece mode.
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
def pair_tiles():
    h = cb.handle()
    h.set_gemm_tile(256, 256, 0)
    yield h
    h.set_gemm_tile(0, 0, 0)
    cb.set_gemm_mode(cb.GemmMode.NATIVE)


def test_pair_config_reported(cuda, pair_tiles):
    assert pair_tiles.gemm_tile(3, 0, 0, 1000, 1000, 1000) == (256, 256, 1)
    pair_tiles.set_gemm_tile(256, 256, 4)
    assert pair_tiles.gemm_tile(3, 0, 0, 1000, 1000, 1000) == (256, 256, 4)
    with pytest.raises(cb.CoralError):
        pair_tiles.set_gemm_tile(256, 128, 0)


SHAPES = [(1, 1, 1), (5, 7, 4), (100, 300, 64), (128, 256, 64), (129, 257, 65), (256, 512, 200),
          (300, 77, 513), (1000, 1000, 1000), (520, 2100, 96)]


@pytest.mark.parametrize("mode,tol", MODES)
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("ops", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_sgemm_pair_random(cuda, mode, tol, shape, ops):
    cb.set_gemm_mode(mode)
    m, n, k = shape
    sample = 4096 if m * n > 100000 else None
    for alpha, beta in [(1.5, 0.5), (1.0, 0.0), (-0.3, 1.0)]:
        gemm_case(cb.sgemm, np.float32, *ops, m, n, k, alpha, beta, tol, sample=sample)


@pytest.mark.parametrize("splits", [2, 3, 8])
@pytest.mark.parametrize("shape", [(256, 256, 2048), (300, 520, 4100)])
def test_sgemm_pair_split_k(cuda, pair_tiles, splits, shape):
    cb.set_gemm_mode(cb.GemmMode.SPLIT_BF16X3)
    pair_tiles.set_gemm_tile(256, 256, splits)
    m, n, k = shape
    gemm_case(cb.sgemm, np.float32, 0, 0, m, n, k, 1.5, 0.5, 4e-5, sample=4096)


@pytest.mark.parametrize("group", [1, 3, 64])
def test_sgemm_pair_raster_groups(cuda, pair_tiles, group):
    cb.set_gemm_mode(cb.GemmMode.SPLIT_BF16X3)
    pair_tiles.set_pair_raster(group)
    try:
        gemm_case(cb.sgemm, np.float32, 1, 0, 1100, 1300, 300, 1.5, 0.5, 4e-5, sample=4096)
    finally:
        pair_tiles.set_pair_raster(0)


@pytest.mark.parametrize("mode,tol", MODES)
@pytest.mark.parametrize("shape", [(5, 7, 4), (127, 129, 65), (300, 260, 700)])
@pytest.mark.parametrize("ops", [(0, 0), (1, 2), (2, 1)])
def test_cgemm_pair_4m(cuda, mode, tol, shape, ops):
    cb.set_gemm_mode(mode)
    m, n, k = shape
    sample = 4096 if m * n > 50000 else None
    gemm_case(cb.cgemm, np.complex64, *ops, m, n, k, 1.5 - 0.5j, 0.25 + 1j, 2 * tol, sample=sample)


def test_sgemm_pair_4096_meets_1e6(cuda):
    """4096^3 NN on pair tiles: component-wise error on 2048 sampled entries
    within the headline bound."""
    m = n = k = 4096
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    A = torch.empty(m * k, device="cuda").uniform_(-1, 1, generator=g)
    B = torch.empty(k * n, device="cuda").uniform_(-1, 1, generator=g)
    C0 = torch.empty(m * n, device="cuda").uniform_(-1, 1, generator=g)
    C = C0.clone()
    cb.set_gemm_mode(cb.GemmMode.SPLIT_BF16X3)
    cb.sgemm(0, 0, m, n, k, 1.5, A, m, B, k, 0.5, C, m)
    torch.cuda.synchronize()
    rng = np.random.default_rng(4)
    ii, jj = rng.integers(0, m, 2048), rng.integers(0, n, 2048)
    want, bound = oracle.gemm_sample(0, 0, m, n, k, 1.5, A.cpu().numpy(), m, B.cpu().numpy(), k, 0.5,
                                     C0.cpu().numpy(), m, ii, jj)
    got = C.cpu().numpy()[ii + jj * m].astype(np.float64)
    assert float((np.abs(got - want) / bound).max()) <= 1e-6


@pytest.mark.parametrize("ops", [(0, 0), (2, 1)])
def test_cgemm_pair_3m(cuda, pair_tiles, ops):
    """3M mapping on pair tiles: the three real split GEMMs each run as
    CTA-pair tiles; tolerance as in the single-CTA 3M tests."""
    cb.set_gemm_mode(cb.GemmMode.SPLIT_BF16X3)
    pair_tiles.set_complex_mapping(1)
    try:
        gemm_case(cb.cgemm, np.complex64, *ops, 300, 260, 700, 1.5 - 0.5j, 0.25 + 1j, 6 * 4e-5, sample=4096)
    finally:
        pair_tiles.set_complex_mapping(0)
