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


def parity_errors(a, b, floor_frac=1e-6):
    """Both error measures of a parity comparison of one field component:
    field  = max |a - b| / max |b|  (the bound the parity tests assert), and
    entry  = max |a - b| / |b| over the entries with |b| >= floor_frac * max |b| (each entry
             against its own size; entries below the floor are rounding-level cancellations of
             much larger terms and have no meaningful relative error of their own)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    if not b.size:
        return 0.0, 0.0
    s = max(np.max(np.abs(b)), np.finfo(float).tiny)
    d = np.abs(a - b)
    field = float(np.max(d) / s)
    m = np.abs(b) >= floor_frac * s
    entry = float(np.max(d[m] / np.abs(b[m]))) if np.any(m) else 0.0
    return field, entry


def record_parity(name, **values):
    """Append one line of measured parity errors to $EWG_PARITY_REPORT (JSON lines), if set."""
    path = os.environ.get("EWG_PARITY_REPORT")
    if not path:
        return
    import json
    with open(path, "a") as f:
        f.write(json.dumps({"test": name, **{k: float(v) if np.isscalar(v) else v for k, v in values.items()}}) + "\n")
