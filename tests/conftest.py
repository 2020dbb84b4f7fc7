"""Shared test setup: import paths, the `gpu` marker, golden-fixture loading.

`-m "not gpu"` runs the oracle-vs-reference checks, host logic and C-ABI
loading on CPU; `-m gpu` runs the CUDA parity tests on a B200.
"""

import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(REPO, "3d-plfbs-gpu_b200"), os.path.join(REPO, "oracle"),
          os.path.join(REPO, "tests", "golden"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


@pytest.fixture(scope="session")
def plfbs_lib():
    from plfbs import build, capi
    build.build()
    return capi.lib()


def load_golden(name):
    d = np.load(os.path.join(REPO, "tests", "golden", name + ".npz"))
    return {k: d[k] for k in d.files}


def rel_err(a, b):
    """max |a - b| / max |b| (0 when both vanish)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max() if b.size else 0.0
    num = np.abs(a - b).max() if b.size else 0.0
    return 0.0 if num == 0 else num / max(den, 1e-300)


def rel_l2(a, b):
    """||a - b||_2 / ||b||_2, the parity measure of the FP64 path."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / max(nb, 1e-300))
