"""Host-side logic of the autotuner/selector (no GPU): shape generation and the
feature vector the library computes for (shape, configuration)."""
import numpy as np

from coral_b200 import tuning


def test_generate_shapes_seeded_and_special():
    a = tuning.generate_shapes(100, seed=1)
    b = tuning.generate_shapes(100, seed=1)
    np.testing.assert_array_equal(a, b)
    assert tuple(a[0]) == (65536, 64, 4096, 0, 0, 3)      # tall-skinny
    assert tuple(a[1]) == (256, 256, 65536, 0, 0, 3)      # split-K heavy
    dims = a[2:, :3]
    assert dims.min() >= 32 and dims.max() <= 16384
    assert set(np.unique(a[:, 3:5])) <= {0, 1}
    assert set(np.unique(a[:, 5])) == {3, 6}              # both split modes


def test_features_shape_and_monotone():
    f = tuning.features((1024, 2048, 4096, 1, 0), 128, 256, 4)
    assert f.shape == (tuning.N_FEATURES,) and np.isfinite(f).all()
    np.testing.assert_allclose(f[:3], np.log2([1024, 2048, 4096]) / 16, rtol=1e-6)
    assert f[3] == 1.0 and f[4] == 0.0
    # tile area relative to 128 x 256: 0.5, 1, 2 (CTA pair)
    assert tuning.features((1024, 2048, 4096, 0, 0), 128, 128, 4)[8] == 0.5
    assert tuning.features((1024, 2048, 4096, 0, 0), 256, 256, 4)[8] == 2.0
    # the 3-piece mode shows in the data-type feature
    assert tuning.features((1024, 2048, 4096, 0, 0, 6), 128, 128, 1)[5] == 1.0
    # more splits -> more work items -> larger occupancy feature
    assert tuning.features((256, 256, 65536, 0, 0), 128, 256, 16)[11] > \
        tuning.features((256, 256, 65536, 0, 0), 128, 256, 1)[11]
    # a pair tile counts against 74 resident pairs, not 148 CTAs
    np.testing.assert_allclose(tuning.features((4096, 4096, 1024, 0, 0), 256, 256, 1)[11],
                               min(256 / 74, 8) / 8, rtol=1e-6)


def test_default_choice_splits_k_for_few_tiles():
    assert tuning.CANDIDATES[tuning.default_choice((256, 256, 65536, 0, 0))] == (128, 256, 16)
    assert tuning.CANDIDATES[tuning.default_choice((8192, 8192, 8192, 0, 0))] == (256, 256, 1)
    assert tuning.CANDIDATES[tuning.default_choice((2048, 2048, 2048, 0, 0))] == (128, 256, 1)
    assert tuning.CANDIDATES[tuning.default_choice((2048, 2048, 2048, 0, 0, 6))] == (128, 128, 1)


def test_candidates_and_validity():
    assert len(tuning.CANDIDATES) == 15
    x6 = (1000, 1000, 1000, 0, 0, 6)
    assert sum(tuning.valid(x6, c) for c in tuning.CANDIDATES) == 10
    assert not tuning.valid(x6, (128, 256, 1)) and tuning.valid(x6, (256, 256, 1))
    shapes = np.array([x6, (1000, 1000, 1000, 0, 0, 3)])
    pred = np.zeros((2, 15))
    pred[:, 5] = -1.0   # a 128 x 256 configuration predicted fastest
    choice = tuning.choose(pred, shapes)
    assert choice[1] == 5 and tuning.valid(shapes[0], tuning.CANDIDATES[choice[0]])


def test_regret_definition():
    t = np.array([[1.0, 2.0], [4.0, 2.0]])
    np.testing.assert_allclose(tuning.regret(t, np.array([0, 0])), [0.0, 1.0])


def test_selector_features_reject_bad_arguments():
    """The feature entry points need no device; they refuse sides past
    INT_MAX (not supported, as the GEMM entry points) and non-positive tile
    widths or split counts (invalid), instead of returning inf/NaN
    features."""
    import ctypes

    from coral_b200 import _lib
    lib = _lib.load()
    out = (ctypes.c_float * 13)()
    ok, invalid, unsupported = 0, 1, 5
    assert lib.coral_selector_features_tile(3, 0, 0, 1024, 1024, 1024, 256, 256, 1, out) == ok
    assert all(abs(v) < 10 for v in out)
    assert lib.coral_selector_features_tile(3, 0, 0, 2**31, 1024, 1024, 128, 256, 1, out) == unsupported
    assert lib.coral_selector_features_tile(3, 0, 0, 1024, 1024, 1024, 128, 0, 1, out) == invalid
    assert lib.coral_selector_features_tile(3, 0, 0, 1024, 1024, 1024, 128, 256, 0, out) == invalid
    assert lib.coral_selector_features_tile(3, 0, 0, 1024, 1024, 1024, 64, 256, 1, out) == invalid
    assert lib.coral_selector_features(3, 0, 0, 1024, 1024, 2**40, 256, 1, out) == unsupported
    assert lib.coral_selector_features(3, 0, 0, 1024, 1024, 1024, -1, 1, out) == invalid
