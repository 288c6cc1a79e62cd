"""Shared fixtures.  `gpu`-marked tests need a CUDA device and the built native library;
everything else runs on the CPU (the oracle, host logic, library load and exports)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libopensc_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def ctx():
    import openspacecharge_b200 as osc
    c = osc.Context(0)
    yield c
    c.close()


def normwise(a, ref, axis=None):
    """max|a-ref| / max|ref| (per component when axis is given)."""
    a = np.asarray(a)
    ref = np.asarray(ref)
    if axis is None:
        return float(np.abs(a - ref).max() / np.abs(ref).max())
    diff = np.abs(a - ref).reshape(-1, ref.shape[axis]) if axis == -1 else None
    return float((diff.max(0) / np.abs(ref).reshape(-1, ref.shape[-1]).max(0)).max())


def rms_rel(a, ref):
    a = np.asarray(a)
    ref = np.asarray(ref)
    return float(np.sqrt(np.mean((a - ref) ** 2)) / np.sqrt(np.mean(ref ** 2)))


def field_err(a, ref):
    """Per-component normwise max and RMS relative error of (..., 3) fields; returns the worst."""
    a = np.asarray(a).reshape(-1, 3)
    ref = np.asarray(ref).reshape(-1, 3)
    mx = max(float(np.abs(a[:, c] - ref[:, c]).max() / np.abs(ref[:, c]).max()) for c in range(3))
    rm = max(rms_rel(a[:, c], ref[:, c]) for c in range(3))
    return mx, rm
