"""Learned tile-width policy of the tensor-core grouped GEMM
(coral_select_grouped_config): the network scores each allowed width for
every instance class present in a batch and installs the argmin.

No reference counterpart.  Checked here: the chosen widths are allowed for
their class, classes without instances keep the handle's width, the result is
what the network's own forward pass over coral_grouped_features predicts, and
a batch run under the chosen policy still matches the oracle.
"""
import ctypes as C
import os

import numpy as np
import pytest
import torch

import coral_b200 as cb
import oracle
from coral_b200 import _lib, tuning

pytestmark = pytest.mark.gpu


def host_records(insts):
    rec = np.zeros(len(insts), dtype=cb.sgemm_problem_dtype())
    for i, (op_a, op_b, m, n, k) in enumerate(insts):
        rec[i] = (op_a, op_b, m, n, k, 1.0, 0.0, 0, 0, 0, 0, m if op_a == 0 else k, k if op_b == 0 else n, m)
    return rec


def select(net, it, rec):
    lib = _lib.load()
    h = cb.handle()
    out = (C.c_int * 4)()
    st = lib.coral_select_grouped_config(h.h, net.p, it, len(rec), rec.ctypes.data_as(C.c_void_p), out)
    assert st == 0, st
    return list(out)


def net_under_test():
    path = os.path.join(tuning.DATA_DIR, "grouped_selector.npz")
    return tuning.Mlp.load(path) if os.path.exists(path) else tuning.Mlp(seed=3)


def test_select_matches_network_argmin(cuda):
    net = net_under_test()
    rng = np.random.default_rng(5)
    insts = [(int(rng.integers(0, 2)), 0, int(m), int(n), int(k))
             for m, n, k in np.exp(rng.uniform(np.log(16), np.log(1024), (500, 3))).astype(int)]
    rec = host_records(insts)
    try:
        for it in (0, 1):
            got = select(net, it, rec)
            assert cb.grouped_config() == got
            for c in range(4):
                members = [x for x in insts if (x[3] <= 64, x[3] <= 128, x[3] <= 256, True).index(True) == c]
                widths = tuning.GROUPED_CLASS_WIDTHS[c]
                assert got[c] in widths
                if not members:
                    continue
                b = len(members)
                m = int(np.sort([x[2] for x in members])[b // 2])
                n = int(np.sort([x[3] for x in members])[b // 2])
                k = int(np.sort([x[4] for x in members])[b // 2])
                op_a = int(2 * sum(x[0] for x in members) > b)
                X = np.stack([tuning.grouped_feature((it, op_a, 0, m, n, k, b), w) for w in widths])
                pred = net.forward(torch.from_numpy(X).cuda()).cpu().numpy().ravel()
                assert got[c] == widths[int(pred.argmin())], (c, got, pred)
    finally:
        cb.set_grouped_config(None)


def test_select_keeps_width_of_empty_classes(cuda):
    net = net_under_test()
    cb.set_grouped_config((128, 64, 256, 64))
    try:
        got = select(net, 1, host_records([(0, 0, 100, 40, 100)] * 10))   # only class 0 present
        assert got[1:] == [64, 256, 64]
        assert got[0] in (64, 128)
    finally:
        cb.set_grouped_config(None)


def test_batch_under_selected_policy_matches_oracle(cuda):
    net = net_under_test()
    rng = np.random.default_rng(9)
    insts, host, keep = [], [], []
    for _ in range(60):
        m, n, k = (int(v) for v in np.exp(rng.uniform(np.log(16), np.log(600), 3)))
        op_a = int(rng.integers(0, 2))
        lda = m if op_a == 0 else k
        a = rng.uniform(-1, 1, lda * (k if op_a == 0 else m)).astype(np.float32)
        b = rng.uniform(-1, 1, k * n).astype(np.float32)
        A = torch.from_numpy(a).cuda().to(torch.bfloat16)
        B = torch.from_numpy(b).cuda().to(torch.bfloat16)
        Cd = torch.zeros(m * n, device="cuda")
        insts.append((op_a, 0, m, n, k))
        host.append((op_a, m, n, k, A.float().cpu().numpy(), lda, B.float().cpu().numpy()))
        keep += [A, B, Cd]
    rec = host_records(insts)
    select(net, 1, rec)
    for i in range(len(insts)):
        rec["a"][i] = keep[3 * i].data_ptr()
        rec["b"][i] = keep[3 * i + 1].data_ptr()
        rec["c"][i] = keep[3 * i + 2].data_ptr()
    desc = torch.from_numpy(rec.view(np.uint8)).cuda()
    try:
        cb.sgemm_grouped(1, len(insts), desc)
        torch.cuda.synchronize()
    finally:
        cb.set_grouped_config(None)
    for i, (op_a, m, n, k, a, lda, b) in enumerate(host):
        got = keep[3 * i + 2].cpu().numpy().reshape(n, m).T
        ii, jj = rng.integers(0, m, 64), rng.integers(0, n, 64)
        want, bound = oracle.gemm_sample(op_a, 0, m, n, k, 1.0, a, lda, b, k, 0.0, np.zeros(m * n, np.float32),
                                         m, ii, jj)
        assert (np.abs(got[ii, jj] - want) <= 4e-5 * bound + 1e-30).all(), i
