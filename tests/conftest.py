"""Shared fixtures.  Marker ``gpu``: needs a CUDA device (B200); every other
test runs on the CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the libgamdb200 kernels)")


def golden(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def rel_rms(got, ref):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    return float(np.sqrt(np.mean((got - ref) ** 2) / np.mean(ref ** 2)))


def sorted_rows(nbl):
    """gamdpy-layout list -> (counts, concatenated per-row sorted ids)."""
    counts = nbl[:, -1].astype(np.int64)
    return counts, np.concatenate([np.sort(nbl[i, : counts[i]]) for i in range(len(nbl))])


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O
