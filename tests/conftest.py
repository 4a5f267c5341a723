import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a library)")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """The CPU oracle is test infrastructure; build it if a checkout lacks it."""
    so = ROOT / "oracle" / "_ref" / "liblbm_oracle.so"
    if not so.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True,
                       stdout=subprocess.DEVNULL)
    yield


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
