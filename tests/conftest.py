"""Shared fixtures: golden data from the reference, the oracle, GPU gating."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def ref_ops(N, variant):
    """The reference's own FP32 operators (tests/golden/ops_N*.npz) with the
    WADG pair of the chosen basis under Vq / Pq."""
    o = golden("ops_N%d.npz" % N)
    o["Vq"], o["Pq"] = o["Vq_" + variant], o["Pq_" + variant]
    return o
