"""The trained selector (coral_b200/data/selector.npz) against exhaustive
autotuning on the 2000 held-out shapes of coral_b200/data/timings_heldout.npz
(every configuration -- CTA-pair 256 x 256, 128 x 256 and 128 x 128 tiles,
each with split-K 1..16 -- timed on a B200 by coral_autotune_sgemm_tiles; a
quarter of the shapes in the 3-piece mode, which has no 128 x 256 tile).

CPU: predictions from the float64 restatement of the network (oracle);
GPU: predictions from the library's own forward kernel.  Both must give a
mean regret <= 5% and beat the default rule (the method without the network).
"""
import os

import numpy as np
import pytest

from coral_b200 import tuning
from oracle import mlp_ref

DATA = tuning.DATA_DIR


def _load():
    d = np.load(os.path.join(DATA, "timings_heldout.npz"))
    w = np.load(os.path.join(DATA, "selector.npz"))
    return d["shapes"], d["times"], w


def test_selector_regret_cpu_oracle():
    shapes, times, w = _load()
    i, h, o = (int(v) for v in w["shape"])
    X = tuning.feature_matrix(shapes)
    y, _ = mlp_ref.forward(w["params"], X, i, h, o)
    choice = tuning.choose(y, shapes)
    r = tuning.regret(times, choice)
    dflt = tuning.regret(times, np.array([tuning.default_choice(s) for s in shapes]))
    assert r.mean() <= 0.05, r.mean()
    assert r.mean() < 0.5 * dflt.mean(), (r.mean(), dflt.mean())


def test_timing_db_is_exhaustive_and_positive():
    shapes, times, _ = _load()
    assert times.shape == (len(shapes), len(tuning.CANDIDATES)) and (times > 0).all()
    # exactly the configurations a shape's mode lacks are +inf
    assert (np.isfinite(times) == tuning.valid_mask(shapes)).all()
    train = np.load(os.path.join(DATA, "timings_train.npz"))
    assert train["times"].shape == (20000, 15)
    # both modes occur, and the pair tiles win on a share of the shapes
    assert set(np.unique(train["shapes"][:, 5])) == {3, 6}
    best = np.array(tuning.CANDIDATES)[train["times"].argmin(1)]
    assert 0.05 < (best[:, 0] == 256).mean() < 0.95
    # held-out shapes come from a different seed than the training shapes
    assert not np.array_equal(train["shapes"][2:12], shapes[2:12])


@pytest.mark.gpu
def test_selector_regret_gpu_kernels(cuda):
    shapes, times, _ = _load()
    net = tuning.Mlp.load(os.path.join(DATA, "selector.npz"))
    choice = tuning.predict_choice(net, shapes)
    r = tuning.regret(times, choice)
    assert r.mean() <= 0.05, r.mean()


# ---- grouped GEMM tile-width network ------------------------------------------
def _load_grouped():
    d = np.load(os.path.join(DATA, "grouped_timings_heldout.npz"))
    w = np.load(os.path.join(DATA, "grouped_selector.npz"))
    return d["samples"], d["times"], w


def _default_width(sample):
    n = int(sample[4])
    return (64, 128, 128, 256)[0 if n <= 64 else 1 if n <= 128 else 2 if n <= 256 else 3]


def test_grouped_selector_regret_cpu_oracle():
    """The grouped network on 1000 held-out uniform batches (seed 13; every
    width timed on a B200): the width it predicts fastest against the measured
    best, from the float64 restatement of the network.  It must stay within 5%
    on average and beat the default per-class widths."""
    samples, times, w = _load_grouped()
    i, h, o = (int(v) for v in w["shape"])
    choice = tuning.predict_grouped_choice(lambda X: mlp_ref.forward(w["params"], X, i, h, o)[0], samples)
    r = tuning.regret(times, choice)
    dflt = tuning.regret(times, np.array([tuning.GROUPED_WIDTHS.index(_default_width(s)) for s in samples]))
    assert r.mean() <= 0.05, r.mean()
    assert r.mean() < dflt.mean(), (r.mean(), dflt.mean())


def test_grouped_timing_db_shape():
    samples, times, _ = _load_grouped()
    assert times.shape == (len(samples), len(tuning.GROUPED_WIDTHS)) and (times > 0).all()
    train = np.load(os.path.join(DATA, "grouped_timings_train.npz"))
    assert train["times"].shape == (6000, 3)
    # both data types and a range of instance counts are present
    assert set(np.unique(train["samples"][:, 0])) == {0, 1}
    assert train["samples"][:, 6].min() == 1 and train["samples"][:, 6].max() > 1000
