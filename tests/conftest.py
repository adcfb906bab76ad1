"""Shared test fixtures.  GPU tests are marked ``gpu`` and run on a B200."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def normalized_error(g, r, nf):
    """max over DOFs of |g - r| / max(|r|, ||r_field||_inf), per field.

    The floor ||r_field||_inf makes the metric meaningful where dudt ~ 0 is the
    result of O(1) cancelling terms summed in a different order.
    """
    g = np.asarray(g).reshape(nf, -1)
    r = np.asarray(r).reshape(nf, -1)
    if not (np.isfinite(g).all() and np.isfinite(r).all()):
        return float("inf")   # a NaN must never compare as small
    out = []
    for f in range(nf):
        scale = np.maximum(np.abs(r[f]), np.abs(r[f]).max())
        scale = np.where(scale == 0, 1.0, scale)
        out.append(float(np.max(np.abs(g[f] - r[f]) / scale)))
    return max(out)


@pytest.fixture(scope="session")
def oracle_mod():
    import pyoracle
    pyoracle.lib()
    return pyoracle
