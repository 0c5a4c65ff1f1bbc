import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running case")


def _ensure_oracle():
    import pyoracle
    if not os.path.exists(pyoracle.LIB_ORACLE) or (
            os.path.isdir(pyoracle.REFERENCE_DIR) and not pyoracle.ref_available()):
        pyoracle.build(ref=True)
    return pyoracle


@pytest.fixture(scope="session")
def po():
    """The test oracle (oracle/pyoracle.py), built on demand."""
    return _ensure_oracle()


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "reference_kernels.npz"))


def _gpu_available() -> bool:
    try:
        r = subprocess.run(["nvidia-smi", "-L"], capture_output=True, text=True, timeout=30)
        return r.returncode == 0 and "GPU" in r.stdout
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda_lib():
    """The product library; built in-tree if missing.  GPU tests only."""
    if not _gpu_available():
        pytest.skip("no CUDA GPU")
    from particlebase_b200 import build as B
    B.build()
    from particlebase_b200 import _lib
    return _lib.lib()
