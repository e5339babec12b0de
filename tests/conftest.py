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

GOLDEN_DECKS = ["small1", "small4", "cap1", "curv1", "grad1", "nucvol1", "am1", "amsub4"]


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


def setup_golden_substrate(target, name: str) -> int:
    """Pre-fills the columnar substrate a golden deck was recorded with (the
    reference got it through MMSREF_INJECT_SUBSTRATE): grains 1..n with their
    rotations, their ids in interior planes 1..top and fs = 1 there.  target:
    a mumatscale_b200.Domain or a tests._oracle.Oracle before its first step.
    Returns n (0 when the deck has no substrate)."""
    rec = golden(name).get("substrate")
    if not rec:
        return 0
    import hashlib
    import mumatscale_b200 as M
    from mumatscale_b200 import workloads as W
    p = M.read_deck(golden_deck(name))
    gx, gy = p.gnsbx * p.gsdimx, p.gnsby * p.gsdimy
    cols, rot = W.columnar_columns(gx, gy, p.cellSize, rec["mean_width"], rec["seed"])
    # the same substrate as the recording (seeded generator)
    assert hashlib.sha256(cols.astype("<i4").tobytes()).hexdigest() == rec["cols"]
    assert hashlib.sha256(rot.astype("<f8").tobytes()).hexdigest() == rec["rotmat"]
    gr = target.download("gr")
    fs = target.download("fs")
    gr[1:rec["top_plane"] + 1, 1:-1, 1:-1] = cols[None]
    fs[gr > 0] = 1.0
    target.set_grains(rot)
    target.upload("gr", gr)
    target.upload("fs", fs)
    return len(rot)


@pytest.fixture(scope="session")
def cuda_device():
    try:
        import torch
        if not torch.cuda.is_available():
            pytest.skip("no CUDA device")
    except Exception:
        pytest.skip("torch unavailable")
    return 0
