"""Shared pytest configuration: the `gpu` marker and helpers for parity tests.

`-m "not gpu"` runs the oracle, golden-fixture and ABI tests on any host;
`-m gpu` runs the CUDA parity tests, which call the kernels through the C ABI
of libcoral_b200.so on an sm_100 device.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU and libcoral_b200.so")


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "golden.npz"))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test collected without a visible CUDA device")
    return torch.device("cuda:0")


def allclose_ref(got, want, rtol, atol):
    """The reference tests' criterion |x-y| <= atol + rtol*max(|x|,|y|)
    (e.g. coral-aarch64/tests/level3/sgemm_tests.rs:64-80)."""
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    assert got.shape == want.shape, (got.shape, want.shape)
    tol = atol + rtol * np.maximum(np.abs(got), np.abs(want))
    bad = np.abs(got - want) > tol
    if bad.any():
        i = int(np.argmax(bad))
        raise AssertionError(f"{int(bad.sum())} mismatches; first at {i}: got {got.flat[i]!r} "
                             f"want {want.flat[i]!r} tol {tol.flat[i]!r}")
