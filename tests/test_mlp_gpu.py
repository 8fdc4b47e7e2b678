"""Split-K / tile-width configurations, the exhaustive autotuner, and the
selector MLP's kernels (no reference counterpart).

The MLP's forward pass and gradients are checked against the float64 numpy
restatement in oracle/mlp_ref.py (relative error <= 1e-4, fp32 kernels vs
fp64 oracle); every configuration of the split-BF16 SGEMM/CGEMM must meet the
split tests' component-wise tolerance.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle
from coral_b200 import _lib, tuning
from oracle import mlp_ref
from test_gemm_gpu import gemm_case

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def restore():
    yield
    h = cb.handle()
    h.lib.coral_set_gemm_tile(h.h, 0, 0, 0)
    h.lib.coral_set_selector(h.h, None)
    cb.set_gemm_mode(cb.GemmMode.NATIVE)


@pytest.mark.parametrize("tm,tn,sp", tuning.CANDIDATES)
def test_split_configs_correct(cuda, tm, tn, sp):
    h = cb.handle()
    assert h.lib.coral_set_gemm_tile(h.h, tm, tn, sp) == 0
    cb.set_gemm_mode(cb.GemmMode.SPLIT_BF16X3)
    gemm_case(cb.sgemm, np.float32, 0, 0, 200, 300, 2000, 1.5, 0.5, 4e-5, sample=2048)
    gemm_case(cb.sgemm, np.float32, 1, 1, 129, 65, 777, 1.0, 0.0, 4e-5)
    gemm_case(cb.cgemm, np.complex64, 2, 1, 70, 90, 333, 1.5 - 0.5j, 0.25 + 1j, 8e-5)
    if (tm, tn) != (128, 256):
        cb.set_gemm_mode(cb.GemmMode.SPLIT_BF16X6)
        gemm_case(cb.sgemm, np.float32, 0, 1, 150, 140, 900, -0.5, 1.0, 1e-5)


def test_split_k_heavy_shape(cuda):
    cb.set_gemm_mode(cb.GemmMode.SPLIT_BF16X3)
    gemm_case(cb.sgemm, np.float32, 0, 0, 256, 256, 65536, 1.0, 0.0, 4e-5, pad=0, sample=1024)


def test_autotune_and_config_restore(cuda):
    h = cb.handle()
    m, n, k = 512, 384, 2048
    A = torch.empty(m * k, device="cuda").uniform_(-1, 1)
    B = torch.empty(k * n, device="cuda").uniform_(-1, 1)
    Cm = torch.empty(m * n, device="cuda")
    ms = (C.c_float * 10)()
    best = C.c_int()
    h.bind_current_stream()
    st = h.lib.coral_autotune_sgemm(h.h, 3, 0, 0, m, n, k, C.c_void_p(A.data_ptr()), m,
                                    C.c_void_p(B.data_ptr()), k, C.c_void_p(Cm.data_ptr()), m, 2, ms,
                                    C.byref(best))
    assert st == 0
    t = np.frombuffer(ms, np.float32)
    assert (t > 0).all() and 0 <= best.value < 10 and t[best.value] == t.min()
    assert cb.gemm_mode() == cb.GemmMode.NATIVE
    bn, sp = C.c_int(), C.c_int()
    assert h.lib.coral_get_gemm_config(h.h, 3, 0, 0, 256, 256, 65536, C.byref(bn), C.byref(sp)) == 0
    assert (bn.value, sp.value) == (256, 16)   # default rule: split K to fill the GPU
    # default rule: CTA-pair tiles once they fill two waves of resident pairs
    assert h.gemm_tile(3, 0, 0, 8192, 8192, 8192) == (256, 256, 1)
    assert h.gemm_tile(3, 0, 0, 2048, 2048, 2048)[0] == 128


def test_autotune_tiles_covers_pair(cuda):
    h = cb.handle()
    m, n, k = 600, 700, 900
    A = torch.empty(m * k, device="cuda").uniform_(-1, 1)
    B = torch.empty(k * n, device="cuda").uniform_(-1, 1)
    Cm = torch.empty(m * n, device="cuda")
    h.bind_current_stream()
    for products, expect in ((3, 15), (6, 10)):
        ms = (C.c_float * 15)()
        count, best = C.c_int(), C.c_int()
        st = h.lib.coral_autotune_sgemm_tiles(h.h, products, 0, 0, m, n, k, C.c_void_p(A.data_ptr()), m,
                                              C.c_void_p(B.data_ptr()), k, C.c_void_p(Cm.data_ptr()), m, 1,
                                              ms, 15, C.byref(count), C.byref(best))
        assert st == 0 and count.value == expect
        t = np.frombuffer(ms, np.float32)[:expect]
        assert (t > 0).all() and t[best.value] == t.min()
    # too small an output array is an argument error, nothing is run
    assert h.lib.coral_autotune_sgemm_tiles(h.h, 3, 0, 0, m, n, k, C.c_void_p(A.data_ptr()), m,
                                            C.c_void_p(B.data_ptr()), k, C.c_void_p(Cm.data_ptr()), m, 1,
                                            ms, 10, C.byref(count), C.byref(best)) == 1
    assert h.gemm_tile(3, 0, 0, 8192, 8192, 8192) == (256, 256, 1)  # configuration restored


def _net_and_batch(seed, batch=64):
    net = tuning.Mlp(seed=seed)
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (batch, tuning.N_FEATURES)).astype(np.float32)
    t = rng.uniform(-1, 1, (batch, 1)).astype(np.float32)
    return net, x, t


def test_mlp_forward_matches_oracle(cuda):
    net, x, t = _net_and_batch(1, batch=300)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    want, _ = mlp_ref.forward(net.get_params(), x, tuning.N_FEATURES, tuning.HIDDEN, 1)
    assert np.abs(y - want).max() <= 1e-4 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("batch", [1, 7, 64, 1000])
def test_mlp_gradients_match_oracle(cuda, batch):
    net, x, t = _net_and_batch(2 + batch, batch)
    g, loss = net.gradients(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    want_loss, want_g = mlp_ref.loss_and_grad(net.get_params(), x, t, tuning.N_FEATURES, tuning.HIDDEN, 1)
    g = g.cpu().numpy().astype(np.float64)
    assert abs(loss - want_loss) <= 1e-4 * abs(want_loss)
    assert np.abs(g - want_g).max() <= 1e-4 * np.abs(want_g).max()


def test_mlp_training_reduces_loss(cuda):
    net = tuning.Mlp(seed=3)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, (4096, tuning.N_FEATURES)).astype(np.float32)
    t = ((x[:, :3] ** 2).sum(1, keepdims=True) - x[:, 3:4]).astype(np.float32)
    X, T = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    first = net.train_step(X, T, 3e-3)
    for _ in range(400):
        last = net.train_step(X, T, 3e-3)
    assert last < 0.05 * first


def test_selector_attached_drives_configuration(cuda):
    h = cb.handle()
    net = tuning.Mlp(seed=4)
    net.attach(h)
    assert h.gemm_tile(3, 0, 0, 1000, 1000, 1000) in tuning.CANDIDATES
    cb.set_gemm_mode(cb.GemmMode.SPLIT_BF16X3)
    gemm_case(cb.sgemm, np.float32, 0, 0, 300, 200, 1500, 1.5, 0.5, 4e-5, sample=2048)
