import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device; runs the sm_100a kernels")


@pytest.fixture
def golden():
    def load(name):
        return dict(np.load(GOLDEN / f"{name}.npz"))

    return load


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def vel_rel_l2(got: dict, ref: dict, keys=("ux", "uy")):
    """Relative L2 error of the velocity vector field (components stacked)."""
    a = np.concatenate([np.asarray(got[k], np.float64).ravel() for k in keys])
    b = np.concatenate([np.asarray(ref[k], np.float64).ravel() for k in keys])
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
