"""The two off-diagonal forms of the SYMV / HEMV / TRMV family against the oracle.

coral_set_strip_form selects the register-streaming strips (default) or the
TMA-fed single pass over the whole triangle (taken when the matrix is 16-byte
aligned with a leading dimension of a multiple of 16 bytes); both must meet
the routines' component-wise bounds (ssymv_tests.rs:152-153 and chemv_tests.rs:190-191:
1e-5 for single precision; 1e-13 for double data) on the same aligned
matrices, with NaN in the unstored triangle.  Sizes cross the 64-column block
and the strip heights (128 rows for float, 64 for double and complex64, 32 for
complex128), with ragged last strips and lda > n.  The TMA form's bounded
waits report a timeout without a fault when the wait limit is set to ~32 ns.
"""
import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle

pytestmark = pytest.mark.gpu

DTS = [np.float32, np.float64, np.complex64, np.complex128]
IDS = ["s", "d", "c", "z"]
TOL = {np.float32: 1e-5, np.float64: 1e-13, np.complex64: 1e-5, np.complex128: 1e-13}
# lda keeps every column 16-byte aligned for all four types
SHAPES = [(64, 64), (130, 132), (300, 300), (1000, 1004), (4100, 4100)]


@pytest.fixture(params=[1, 0], ids=["tma", "register"])
def form(request):
    h = cb.handle()
    h.set_strip_form(request.param)
    yield request.param
    h.set_strip_form(0)


def rnd(rng, shape, dt):
    if np.issubdtype(dt, np.complexfloating):
        return (rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)).astype(dt)
    return rng.uniform(-1, 1, shape).astype(dt)


def tri(rng, n, lda, uplo, dt, nan_diag=False):
    a = rnd(rng, (n, lda), dt)                                   # [col][row]
    jj, ii = np.meshgrid(np.arange(n), np.arange(lda), indexing="ij")
    stored = (ii <= jj) if uplo == 0 else (ii >= jj)
    a[~stored & (ii < n)] = np.nan
    if nan_diag:
        d = np.arange(n)
        a[d, d] = np.nan
    return a


def stored_mag(a, n, uplo):
    A = np.nan_to_num(np.abs(a[:, :n].T.astype(np.complex128)))
    return np.triu(A) if uplo == 0 else np.tril(A)


def check(got, want, scale, dt):
    assert np.isfinite(got).all()
    err = np.abs(got - want)
    assert (err <= TOL[dt] * scale + 1e-30).all(), float((err / (scale + 1e-30)).max())


def symv(dt, uplo, n, alpha, a, lda, x, beta, y):
    A = torch.from_numpy(a.ravel()).cuda()
    X = torch.from_numpy(x).cuda()
    Y = torch.from_numpy(y.copy()).cuda()
    if dt == np.float32:
        cb.ssymv(uplo, n, alpha.real, A, lda, X, 1, beta.real, Y, 1)
        want = oracle.ssymv(uplo, n, alpha.real, a.ravel(), lda, x, 1, beta.real, y, 1)
    elif dt == np.float64:
        cb.dsymv(uplo, n, alpha.real, A, lda, X, 1, beta.real, Y, 1)
        want = oracle.dsymv(uplo, n, alpha.real, a.ravel(), lda, x, 1, beta.real, y, 1)
    elif dt == np.complex64:
        cb.chemv(uplo, n, alpha, A, lda, X, 1, beta, Y, 1)
        w = oracle.chemv(uplo, n, np.array([alpha.real, alpha.imag], np.float32), a.ravel().view(np.float32), lda,
                         x.view(np.float32), 1, np.array([beta.real, beta.imag], np.float32),
                         y.view(np.float32), 1)
        want = w[0::2] + 1j * w[1::2]
    else:
        cb.zhemv(uplo, n, alpha, A, lda, X, 1, beta, Y, 1)
        want = oracle.zhemv(uplo, n, alpha, a.ravel(), lda, x, 1, beta, y, 1)
    torch.cuda.synchronize()
    return Y.cpu().numpy(), want


@pytest.mark.parametrize("dt", DTS, ids=IDS)
@pytest.mark.parametrize("n,lda", SHAPES)
@pytest.mark.parametrize("uplo", [0, 1])
def test_symv_hemv_both_forms(cuda, form, dt, n, lda, uplo):
    rng = np.random.default_rng(n + 3 * uplo + 17 * DTS.index(dt))
    a = tri(rng, n, lda, uplo, dt)
    x, y = rnd(rng, n, dt), rnd(rng, n, dt)
    cplx = np.issubdtype(dt, np.complexfloating)
    alpha = np.complex128(1.5 - 0.5j if cplx else 1.5)
    beta = np.complex128(0.25 + 0.5j if cplx else 0.5)
    got, want = symv(dt, uplo, n, alpha, a, lda, x, beta, y)
    M = stored_mag(a, n, uplo)
    full = M + M.T - np.diag(np.diag(M))
    check(got, want, abs(alpha) * full @ np.abs(x) + abs(beta) * np.abs(y), dt)


@pytest.mark.parametrize("dt", DTS, ids=IDS)
@pytest.mark.parametrize("n,lda", [(300, 300), (4100, 4100)])
@pytest.mark.parametrize("uplo", [0, 1])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_trmv_both_forms(cuda, form, dt, n, lda, uplo, trans):
    rng = np.random.default_rng(n + 7 * uplo + 11 * trans)
    # unit diagonal (CORAL_UNIT = 0; NaN stored there must not be read) for N and C, non-unit for T
    diag = 1 if trans == 1 else 0
    a = tri(rng, n, lda, uplo, dt, nan_diag=(diag == 0))
    x = rnd(rng, n, dt)
    X = torch.from_numpy(x.copy()).cuda()
    fn = {np.float32: cb.strmv, np.float64: cb.dtrmv, np.complex64: cb.ctrmv, np.complex128: cb.ztrmv}[dt]
    fn(uplo, trans, diag, n, torch.from_numpy(a.ravel()).cuda(), lda, X, 1)
    torch.cuda.synchronize()
    orc = {np.float32: oracle.strmv, np.float64: oracle.dtrmv, np.complex64: oracle.ctrmv,
           np.complex128: oracle.ztrmv}[dt]
    want = orc(uplo, trans, diag, n, a.ravel(), lda, x, 1)
    M = stored_mag(a, n, uplo)
    if diag == 0:
        np.fill_diagonal(M, 1.0)
    check(X.cpu().numpy(), want, (M if trans == 0 else M.T) @ np.abs(x), dt)


def test_forms_agree_at_8192(cuda):
    """SSYMV upper n = 8192 (the benchmarked configuration) in both forms:
    each within the bound of the oracle, and within rounding of each other."""
    n = 8192
    rng = np.random.default_rng(8192)
    a = tri(rng, n, n, 0, np.float32)
    x, y = rnd(rng, n, np.float32), rnd(rng, n, np.float32)
    h = cb.handle()
    outs = []
    try:
        for f in (1, 0):
            h.set_strip_form(f)
            got, want = symv(np.float32, 0, n, np.complex128(1.5), a, n, x, np.complex128(0.5), y)
            M = stored_mag(a, n, 0)
            scale = 1.5 * ((M + M.T - np.diag(np.diag(M))) @ np.abs(x)) + 0.5 * np.abs(y)
            check(got, want, scale, np.float32)
            outs.append(got)
    finally:
        h.set_strip_form(0)
    assert np.abs(outs[0] - outs[1]).max() <= 2e-5 * np.abs(outs[1]).max()


def test_tma_form_wait_timeout_reports_status(cuda):
    """With a wait limit of ~32 ns the consumers' first waits on the TMA ring
    give up before the copies land: the status word is set, the CTAs drain
    their copies and exit, coral_sync reports CORAL_ERR_TIMEOUT, and the next
    call (default limit) is correct."""
    n = 4096
    rng = np.random.default_rng(4096)
    a = tri(rng, n, n, 1, np.float32)
    x, y = rnd(rng, n, np.float32), rnd(rng, n, np.float32)
    h = cb.handle()
    A = torch.from_numpy(a.ravel()).cuda()
    X = torch.from_numpy(x).cuda()
    h.set_strip_form(1)
    h.set_wait_limit(1)
    try:
        cb.ssymv(1, n, 1.0, A, n, X, 1, 0.0, torch.zeros(n, device="cuda"), 1)
        with pytest.raises(cb.CoralError) as e:
            h.sync()
        assert e.value.status == 3
    finally:
        h.set_wait_limit(0)
    try:
        got, want = symv(np.float32, 1, n, np.complex128(1.0), a, n, x, np.complex128(0.0), y)
    finally:
        h.set_strip_form(0)
    M = stored_mag(a, n, 1)
    check(got, want, (M + M.T - np.diag(np.diag(M))) @ np.abs(x), np.float32)
