import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running oracle comparison")


@pytest.fixture(scope="session", autouse=True)
def built():
    """Builds the product library and the oracles once per session (in-tree)."""
    from astaroth_b200 import build as b
    b.build()
    # the reference model (oracle/_ref) is built where the reference tree is
    # found: $AC_REFERENCE, else a checkout named "reference" beside the repository
    ref = os.environ.get("AC_REFERENCE")
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")] + ([f"REF={ref}"] if ref else []),
                   check=True)
    yield


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
