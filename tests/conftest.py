"""Shared test setup: the `gpu` marker, import paths and small helpers.

Tests marked `gpu` need a CUDA device and the built libmhdgpu.so; the others
run on CPU.  The oracle (oracle/mhd_oracle.py, oracle/ref.py) is imported
here only as the checker.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built libmhdgpu.so")
    config.addinivalue_line("markers", "slow: long-running")


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def rel_l2(a, b):
    """Per-field relative L2 error of a against b; fields whose reference norm
    is tiny use the norm of the whole state as the scale."""
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.linalg.norm(b)
    out = []
    for v in range(b.shape[0]):
        den = np.linalg.norm(b[v])
        if den < 1e-8 * scale:
            den = scale
        out.append(float(np.linalg.norm(a[v] - b[v]) / den))
    return np.array(out)


def rel_l2_own(a, b):
    """Per-field relative L2 error of a against b, each field measured against
    its own norm only; a field that is identically zero in b must be
    identically zero in a (error 0, else inf)."""
    a = np.asarray(a)
    b = np.asarray(b)
    out = []
    for v in range(b.shape[0]):
        den = np.linalg.norm(b[v])
        num = np.linalg.norm(a[v] - b[v])
        out.append(float(num / den) if den > 0 else (0.0 if num == 0 else float("inf")))
    return np.array(out)


@pytest.fixture(scope="session")
def reference():
    import ref
    if not ref.available():
        if ref.sources_present():
            ref.build()
        else:
            pytest.skip("reference oracle not built")
    return ref.Reference()
