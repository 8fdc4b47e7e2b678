"""SSYMV, CHEMV, STRMV and STRSV parity through the C ABI.

Against the fp64/double-double oracle with scaled bounds
|err| <= tol * (|alpha| |A||x| + |beta y|) (tol 1e-5: ssymv_tests.rs:152-153,
chemv_tests.rs:190-191) and, for STRSV, the reference's closed-form fixtures
against golden CBLAS outputs with its tolerance 1e-4 (strsv_tests.rs:213-214).
The unstored triangle (and, for unit-diagonal cases, the diagonal) is filled
with NaN: any read of it would show up in the result (chemv_tests.rs:303-447
checks the same "stored triangle + garbage" property).
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import fixtures as fx
import oracle
from conftest import allclose_ref

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def tri_matrix(n, lda, uplo, seed, complex_=False, diag_boost=0.0, garbage_diag=False):
    rng = np.random.default_rng(seed)
    shape = (n, lda)  # [col][row]
    if complex_:
        a = (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(np.complex64)
    else:
        a = rng.uniform(-1, 1, shape).astype(np.float32)
    jj, ii = np.meshgrid(np.arange(n), np.arange(lda), indexing="ij")
    stored = (ii <= jj) if uplo == 0 else (ii >= jj)
    a[~stored & (ii < n)] = np.nan
    d = np.arange(n)
    if diag_boost:
        a[d, d] = a[d, d] + np.float32(diag_boost)
    if garbage_diag:
        a[d, d] = np.nan
    return a.reshape(-1)


SIZES = [(1, 1), (7, 7), (63, 63), (64, 64), (65, 70), (127, 132), (300, 300), (1024, 1024),
         (2049, 2050)]


@pytest.mark.parametrize("n,lda", SIZES)
@pytest.mark.parametrize("uplo", [0, 1])
def test_ssymv(cuda, n, lda, uplo):
    a = tri_matrix(n, lda, uplo, n)
    for (alpha, beta, inc) in [(1.5, 0.5, 1), (1.0, 0.0, 1), (-0.7, 1.0, 2), (0.0, 0.3, 1)]:
        x = np.random.default_rng(1).uniform(-1, 1, (n - 1) * inc + 1).astype(np.float32)
        y = np.random.default_rng(2).uniform(-1, 1, (n - 1) * inc + 1).astype(np.float32)
        Y = dev(y)
        cb.ssymv(uplo, n, alpha, dev(a), lda, dev(x), inc, beta, Y, inc)
        got = host(Y)[::inc][:n]
        want = oracle.ssymv(uplo, n, alpha, a, lda, x, inc, beta, y, inc)
        full = np.nan_to_num(a.reshape(n, lda).T[:n, :].astype(np.float64))
        sym = np.where(np.isnan(a.reshape(n, lda).T[:n, :]), full.T, full)
        scale = abs(alpha) * (np.abs(sym) @ np.abs(x[::inc][:n])) + np.abs(beta * y[::inc][:n])
        assert np.isfinite(got).all()
        assert (np.abs(got - want) <= 1e-5 * scale + 1e-6).all()


@pytest.mark.parametrize("n,lda", SIZES[:-1])
@pytest.mark.parametrize("uplo", [0, 1])
def test_chemv(cuda, n, lda, uplo):
    a = tri_matrix(n, lda, uplo, n, complex_=True)
    d = np.arange(n)
    a2 = a.reshape(n, lda)
    a2[d, d] = a2[d, d].real + 1j * np.float32(123.0)  # imaginary part of the diagonal is ignored
    a = a2.reshape(-1)
    for (alpha, beta, inc) in [((1.5, -0.5), (0.25, 1.0), 1), ((1.0, 0.0), (0.0, 0.0), 1),
                               ((0.5, 0.5), (1.0, 0.0), 3)]:
        x = (np.random.default_rng(1).uniform(-1, 1, (n - 1) * inc + 1)
             + 1j * np.random.default_rng(3).uniform(-1, 1, (n - 1) * inc + 1)).astype(np.complex64)
        y = (np.random.default_rng(2).uniform(-1, 1, (n - 1) * inc + 1)
             + 1j * np.random.default_rng(4).uniform(-1, 1, (n - 1) * inc + 1)).astype(np.complex64)
        Y = dev(y)
        cb.chemv(uplo, n, complex(*alpha), dev(a), lda, dev(x), inc, complex(*beta), Y, inc)
        got = host(Y)[::inc][:n]
        w = oracle.chemv(uplo, n, np.array(alpha, np.float32), a.view(np.float32), lda,
                         x.view(np.float32), inc, np.array(beta, np.float32), y.view(np.float32), inc)
        want = w[0::2] + 1j * w[1::2]
        mag = np.abs(np.nan_to_num(a.reshape(n, lda).T[:n, :]))
        mag = np.maximum(mag, mag.T)
        scale = np.hypot(*alpha) * (mag @ np.abs(x[::inc][:n])) + np.hypot(*beta) * np.abs(y[::inc][:n])
        assert np.isfinite(got).all()
        assert (np.abs(got - want) <= 2e-5 * scale + 1e-6).all()


@pytest.mark.parametrize("n,lda", SIZES)
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
@pytest.mark.parametrize("diag", [0, 1])
def test_strmv(cuda, n, lda, uplo, trans, diag):
    a = tri_matrix(n, lda, uplo, n, garbage_diag=(diag == 0))
    inc = 2 if n % 2 else 1
    x = np.random.default_rng(5).uniform(-1, 1, (n - 1) * inc + 1).astype(np.float32)
    X = dev(x)
    cb.strmv(uplo, trans, diag, n, dev(a), lda, X, inc)
    got = host(X)[::inc][:n]
    want = oracle.strmv(uplo, trans, diag, n, a, lda, x, inc)
    assert np.isfinite(got).all()
    mag = np.abs(np.nan_to_num(a.reshape(n, lda).T[:n, :])) + np.eye(n)
    if trans:
        mag = mag.T
    scale = mag @ np.abs(x[::inc][:n])
    assert (np.abs(got - want) <= 1e-5 * scale + 1e-6).all()


def test_strsv_reference_fixtures(cuda, golden):
    for si, (n, lda, incs) in enumerate(fx.TRSV_SHAPES):
        for uplo in (0, 1):
            a = fx.trsv_matrix(n, lda, uplo)
            A = dev(a)
            for inc in incs:
                x = fx.trsv_x(n, inc)
                for trans in (0, 1):
                    for diag in (0, 1):
                        X = dev(x)
                        cb.strsv(uplo, trans, diag, n, A, lda, X, inc)
                        got = host(X)[::inc][:n]
                        allclose_ref(got, golden[f"strsv_s{si}_u{uplo}_i{inc}_t{trans}_d{diag}"],
                                     1e-4, 1e-4)


@pytest.mark.parametrize("n,lda", SIZES + [(4096, 4096)])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("diag", [0, 1])
def test_strsv_random(cuda, n, lda, uplo, trans, diag):
    # diag = n + U[0,1] for conditioning, as in the STRSV n = 4096 bandwidth workload
    a = tri_matrix(n, lda, uplo, n + 11, diag_boost=float(n), garbage_diag=(diag == 0))
    if diag == 0:  # unit diagonal: keep the off-diagonal small so the system stays well posed
        a = np.where(np.isnan(a), a, a / np.float32(max(n, 1)))
    inc = 3 if n == 127 else 1
    x = np.random.default_rng(9).uniform(-1, 1, (n - 1) * inc + 1).astype(np.float32)
    X = dev(x)
    cb.strsv(uplo, trans, diag, n, dev(a), lda, X, inc)
    got = host(X)[::inc][:n]
    want = oracle.strsv(uplo, trans, diag, n, a, lda, x, inc)
    assert np.isfinite(got).all()
    allclose_ref(got, want, 1e-4, 1e-6)
    # untouched stride holes
    if inc > 1:
        holes = np.arange(x.size) % inc != 0
        np.testing.assert_array_equal(host(X)[holes], x[holes])


def test_strsv_repeated_calls_reuse_flags(cuda):
    """Back-to-back solves reuse the ready flags by epoch (no reset pass)."""
    n = 1000
    a = tri_matrix(n, n, 1, 3, diag_boost=float(n))
    A = dev(a)
    x = np.random.default_rng(1).uniform(-1, 1, n).astype(np.float32)
    want = oracle.strsv(1, 0, 1, n, a, n, x, 1)
    for _ in range(5):
        X = dev(x)
        cb.strsv(1, 0, 1, n, A, n, X, 1)
        allclose_ref(host(X), want, 1e-4, 1e-6)
    cb.handle().sync()


def test_strsv_wait_timeout_reports_status(cuda):
    """Failure detection without a GPU fault: with a wait limit of ~32 ns the
    blocks that wait for earlier blocks give up, set the status word and
    exit; coral_sync reports CORAL_ERR_TIMEOUT, the context stays usable and
    the next solve (default limit) is correct."""
    n = 4096
    a = tri_matrix(n, n, 1, 4, diag_boost=float(n))
    A = dev(a)
    x = np.random.default_rng(2).uniform(-1, 1, n).astype(np.float32)
    h = cb.handle()
    h.set_wait_limit(1)
    try:
        cb.strsv(1, 0, 1, n, A, n, dev(x), 1)
        with pytest.raises(cb.CoralError) as e:
            h.sync()
        assert e.value.status == 3
    finally:
        h.set_wait_limit(0)
    X = dev(x)
    cb.strsv(1, 0, 1, n, A, n, X, 1)
    h.sync()
    allclose_ref(host(X), oracle.strsv(1, 0, 1, n, a, n, x, 1), 1e-4, 1e-6)


@pytest.mark.parametrize("layout", ["tma", "odd_lda", "unaligned"])
@pytest.mark.parametrize("n,uplo,trans,diag", [(1000, 1, 0, 1), (1000, 0, 1, 1), (4097, 0, 0, 0),
                                               (4097, 1, 1, 1), (130, 1, 1, 0), (520, 0, 0, 1)])
def test_strsv_both_paths(cuda, layout, n, uplo, trans, diag):
    """The tensor-map path (lda % 4 == 0, 16-byte aligned A) and the plain-load
    path (any other layout) solve the same systems; clusters of 8 blocks with
    ragged last blocks and partial last clusters included."""
    lda = n + (1 if layout == "odd_lda" else (4 - n % 4) % 4)
    a = tri_matrix(n, lda, uplo, n + lda, diag_boost=float(n), garbage_diag=(diag == 0))
    if diag == 0:
        a = np.where(np.isnan(a), a, a / np.float32(n))
    x = np.random.default_rng(lda).uniform(-1, 1, n).astype(np.float32)
    if layout == "unaligned":
        buf = dev(np.concatenate([np.zeros(1, np.float32), a]))
        A = buf[1:]
    else:
        A = dev(a)
    X = dev(x)
    cb.strsv(uplo, trans, diag, n, A, lda, X, 1)
    allclose_ref(host(X), oracle.strsv(uplo, trans, diag, n, a, lda, x, 1), 1e-4, 1e-6)


def test_strsv_graph_replay(cuda):
    """The solve keeps its per-call state (tickets, epoch) on the device, so a
    captured solve replays correctly any number of times."""
    n = 3000
    a = tri_matrix(n, n, 1, 21, diag_boost=float(n))
    A = dev(a)
    x = np.random.default_rng(5).uniform(-1, 1, n).astype(np.float32)
    B = dev(x)
    X = B.clone()
    cb.strsv(1, 0, 1, n, A, n, X, 1)  # first call sizes the slot array outside capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            X.copy_(B)
            cb.strsv(1, 0, 1, n, A, n, X, 1)
    torch.cuda.current_stream().wait_stream(s)
    want = oracle.strsv(1, 0, 1, n, a, n, x, 1)
    for _ in range(4):
        X.fill_(float("nan"))
        g.replay()
        allclose_ref(host(X), want, 1e-4, 1e-6)
    del g
    cb.handle().sync()
