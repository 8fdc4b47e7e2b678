"""Level-1 parity through the C ABI against the oracle (coral-aarch64/src/level1).

Bit-exact: isamax (index), saxpy, sscal, scopy, sswap.  Tolerance (the
reference tests' own): sdot 4e-6 (tests/level1/dot_tests.rs:176-177),
snrm2 1e-6 (nrm2_tests.rs:106-107).
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def rnd(n, seed):
    return np.random.default_rng(seed).uniform(-1, 1, n).astype(np.float32)


SIZES = [1, 3, 7, 8, 15, 16, 17, 1000, 4096 + 3, 1 << 20, (1 << 20) + 5]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [1, 3])
def test_sdot(cuda, n, inc):
    x, y = rnd((n - 1) * inc + 1, n), rnd((n - 1) * inc + 1, n + 1)
    got = cb.sdot(n, dev(x), inc, dev(y), inc)
    want = oracle.sdot(n, x, inc, y, inc)
    assert abs(got - want) <= 4e-6 + 4e-6 * abs(want), (got, want)


def test_sdot_misaligned_and_empty(cuda):
    x, y = rnd(1025, 1), rnd(1025, 2)
    X, Y = dev(x), dev(y)
    got = cb.sdot(1024, X[1:], 1, Y[1:], 1)
    want = oracle.sdot(1024, x[1:].copy(), 1, y[1:].copy(), 1)
    assert abs(got - want) <= 4e-6 + 4e-6 * abs(want)
    assert cb.sdot(0, X, 1, Y, 1) == 0.0


def test_sdot_full_size(cuda):
    n = 1 << 26
    x, y = rnd(n, 11), rnd(n, 12)
    got = cb.sdot(n, dev(x), 1, dev(y), 1)
    want = oracle.sdot(n, x, 1, y, 1)
    assert abs(got - want) <= 4e-6 * max(1.0, abs(want))


@pytest.mark.parametrize("n", SIZES)
def test_snrm2(cuda, n):
    x = rnd(n, n)
    got = cb.snrm2(n, dev(x), 1)
    want = oracle.snrm2(n, x, 1)
    assert abs(got - want) <= 1e-6 * want + 1e-30


def test_snrm2_overflow_safe_and_edges(cuda):
    x = np.array([2e38, 1e38, -1e38], np.float32)  # norm 2.45e38 < FLT_MAX
    got = cb.snrm2(3, dev(x), 1)
    want = oracle.snrm2(3, x, 1)
    assert np.isfinite(got) and abs(got - want) <= 1e-6 * want
    tiny = np.full(64, 1e-40, np.float32)
    assert abs(cb.snrm2(64, dev(tiny), 1) - oracle.snrm2(64, tiny, 1)) <= 1e-6 * 8e-40
    assert cb.snrm2(0, dev(x), 1) == 0.0 and cb.snrm2(3, dev(x), 0) == 0.0
    xs = rnd(3001, 5)
    assert abs(cb.snrm2(1000, dev(xs), 3) - oracle.snrm2(1000, xs, 3)) <= 1e-6 * oracle.snrm2(1000, xs, 3)


def test_isamax_planted_reference_cases(cuda, golden):
    import fixtures as fx
    for ci, (n, inc, x) in enumerate(fx.isamax_cases()):
        assert cb.isamax(n, dev(x), inc) == int(golden[f"isamax_c{ci}"][0])


@pytest.mark.parametrize("n", [5, 16, 17, 1000, (1 << 20) + 3, 1 << 26])
def test_isamax_planted_ties(cuda, n):
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, n).astype(np.float32)
    k = min(5, n)
    idx = np.sort(rng.choice(n, size=k, replace=False))
    x[idx] = np.where(np.arange(k) % 2 == 0, 2.5, -2.5).astype(np.float32)
    got = cb.isamax(n, dev(x), 1)
    assert got == oracle.isamax(n, x, 1) == idx[0]


def test_isamax_nan_inf_strided(cuda):
    x = rnd(3000, 9)
    x[7] = np.nan
    x[100] = -np.inf
    x[2000] = np.inf
    assert cb.isamax(3000, dev(x), 1) == oracle.isamax(3000, x, 1) == 100
    assert cb.isamax(1000, dev(x), 3) == oracle.isamax(1000, x, 3)
    assert cb.isamax(4, dev(np.full(4, np.nan, np.float32)), 1) == 0
    assert cb.isamax(0, dev(x), 1) == 0 and cb.isamax(5, dev(x), 0) == 0
    X = dev(x)
    assert cb.isamax(2999, X[1:], 1) == oracle.isamax(2999, x[1:].copy(), 1)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inc", [(1, 1), (2, 3)])
def test_saxpy_bit_exact(cuda, n, inc):
    ix, iy = inc
    x, y = rnd((n - 1) * ix + 1, n), rnd((n - 1) * iy + 1, n + 7)
    Y = dev(y)
    cb.saxpy(n, 0.37, dev(x), ix, Y, iy)
    np.testing.assert_array_equal(host(Y), oracle.saxpy(n, 0.37, x, ix, y, iy))


def test_saxpy_misaligned_and_quick_returns(cuda):
    x, y = rnd(1031, 1), rnd(1031, 2)
    Y = dev(y)
    cb.saxpy(1030, -1.25, dev(x)[1:], 1, Y[1:], 1)
    want = y.copy()
    want[1:] = oracle.saxpy(1030, -1.25, x[1:].copy(), 1, y[1:].copy(), 1)
    np.testing.assert_array_equal(host(Y), want)
    Y = dev(y)
    cb.saxpy(1031, 0.0, dev(x), 1, Y, 1)
    np.testing.assert_array_equal(host(Y), y)


def test_saxpy_bad_increment(cuda):
    x = dev(rnd(8, 1))
    with pytest.raises(cb.CoralError) as e:
        cb.saxpy(8, 1.0, x, 0, x, 1)
    assert e.value.status == 1 and e.value.bad_arg == 4


@pytest.mark.parametrize("n", [1, 9, 1000, (1 << 20) + 1])
def test_sscal_scopy_sswap_bit_exact(cuda, n):
    x, y = rnd(n, 1), rnd(n, 2)
    X = dev(x)
    cb.sscal(n, 0.3, X, 1)
    np.testing.assert_array_equal(host(X), oracle.sscal(n, 0.3, x, 1))
    X, Y = dev(x), dev(y)
    cb.sswap(n, X, 1, Y, 1)
    np.testing.assert_array_equal(host(X), y)
    np.testing.assert_array_equal(host(Y), x)
    Y = dev(y)
    cb.scopy(n, dev(x), 1, Y, 1)
    np.testing.assert_array_equal(host(Y), x)


def test_strided_copy_swap_scal(cuda):
    x, y = rnd(3 * 500, 1), rnd(2 * 500, 2)
    Y = dev(y)
    cb.scopy(500, dev(x), 3, Y, 2)
    np.testing.assert_array_equal(host(Y), oracle.scopy(500, x, 3, y, 2))
    X, Y = dev(x), dev(y)
    cb.sswap(500, X, 3, Y, 2)
    wx, wy = oracle.sswap(500, x, 3, y, 2)
    np.testing.assert_array_equal(host(X), wx)
    np.testing.assert_array_equal(host(Y), wy)
    X = dev(x)
    cb.sscal(500, 0.0, X, 3)  # sscal multiplies even by zero (sscal.rs:41-51)
    np.testing.assert_array_equal(host(X), oracle.sscal(500, 0.0, x, 3))
