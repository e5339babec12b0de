"""Shared fixtures.  Tests marked ``gpu`` need a B200 and the in-tree CUDA
library; everything else runs on the CPU (the oracle, the host logic, the
library's exports)."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

GOLDEN_DECKS = ["small1", "small4", "cap1", "curv1", "grad1", "nucvol1", "am1"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def built():
    """Builds libmms_b200.so and the oracle library if they are missing."""
    from mumatscale_b200 import build as b
    b.build()
    import subprocess
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True, capture_output=True)
    return True


def golden(name: str) -> dict:
    return json.loads((GOLDEN / f"{name}.json").read_text())


def golden_deck(name: str) -> Path:
    return GOLDEN / golden(name)["deck"]


@pytest.fixture(scope="session")
def cuda_device():
    try:
        import torch
        if not torch.cuda.is_available():
            pytest.skip("no CUDA device")
    except Exception:
        pytest.skip("torch unavailable")
    return 0
