import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a engine)")


@pytest.fixture(scope="session")
def oa():
    import openadmixture_b200
    return openadmixture_b200


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session", params=["small_k3", "small_k5"])
def golden(request):
    return load_golden(request.param)


def rel_err(a, b, scale=None):
    a = np.asarray(a, dtype=np.float64); b = np.asarray(b, dtype=np.float64)
    s = np.abs(b) if scale is None else scale
    return float(np.max(np.abs(a - b) / np.maximum(s, 1e-300)))
