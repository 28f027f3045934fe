"""pytest configuration: the `gpu` marker, import paths and shared fixtures.

Tests marked `gpu` need a B200 and the built libewg.so; everything else runs on CPU. The CPU
oracle (oracle/) is the checker for every parity test.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ewoms-numerics_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device and libewg.so")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def ewg_mod():
    import ewg
    return ewg


def rel_close(a, b, rtol, scale=None):
    """max |a - b| <= rtol * scale, with scale = max |b| unless given (blocks of a field that
    are tiny compared with the field's magnitude are judged against the field, not themselves)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.max(np.abs(b)) if scale is None else scale
    err = np.max(np.abs(a - b)) if a.size else 0.0
    return err <= rtol * max(s, np.finfo(float).tiny), err, s
