"""The command-line driver mmsb200 (a C host over the C ABI) run the way the
reference's regression scripts run muMatScale: ``<exe> -i -c <deck>``, with
their output parsed the same way (tests/testOneGrain.py:25-39 and
tests/testAMtrack.py:25-56 of the reference: the grain count and average
volume from the "Average" line, the fraction solid from the last screen
line), and a restart from the run loop's checkpoint (``-r``,
ca_main.c:136-137)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

import mumatscale_b200 as M
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

EXE = Path(M.__file__).resolve().parent / "mmsb200"


def run_cli(deck: Path, cwd: Path, *extra: str, timeout: float = 600) -> list[bytes]:
    r = subprocess.run([str(EXE), "-i", "-c", str(deck), *extra], cwd=cwd, capture_output=True,
                       timeout=timeout)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    return r.stdout.split(b"\n")


def summary(lines: list[bytes]) -> tuple[int, float]:
    """(grains, average mm^3) from the "Average" line, as the reference's
    scripts read it: words[0] and words[9]."""
    for line in lines:
        if line.count(b"Average"):
            words = line.split()
            return int(words[0]), float(words[9])
    raise AssertionError("no Average line")


def last_fs(lines: list[bytes]) -> float:
    """Fraction solid (percent) of the last screen line between the "Wall"
    header and the "Average" line, as testAMtrack.py reads it."""
    flag, fs = 0, None
    for line in lines:
        # the interactive screen lines start with a carriage return
        line = line.split(b"\r")[-1]
        if line.count(b"Wall"):
            flag = 1
        if line.count(b"Average"):
            flag = 0
        words = line.split()
        if len(words) == 4 and flag > 0:
            fs = float(words[2][:-1])
    assert fs is not None, "no screen line"
    return fs


def test_cli_one_grain(built, cuda_device, tmp_path):
    """testOneGrain.py: 1 grain, average 0.000737875 mm^3 +- 1e-6."""
    ng, avg = summary(run_cli(GOLDEN / "decks" / "one_grain.in", tmp_path))
    assert ng == 1
    assert abs(avg - 0.000737875) <= 1e-6


@pytest.mark.parametrize("form", ["f64", "f32"])
def test_cli_am_track(built, cuda_device, tmp_path, form):
    """testAMtrack.py (am_singletrack.in, 3 x 2 x 1 ranks, 600 steps of the
    moving-source temperature): 1889 grains, average 9.1e-7 mm^3 +- 1e-8,
    fraction solid 86 % +- 0.2.  Both forms meet the reference's own
    tolerances (CUDA's exp is not glibc's, and the FP32 form's temperature
    comes from the tensor cores)."""
    lines = run_cli(GOLDEN / "decks" / "am_singletrack.in", tmp_path, "-p", form)
    ng, avg = summary(lines)
    assert ng == 1889
    assert abs(avg - 9.1e-7) <= 1e-8, avg
    assert abs(last_fs(lines) - 86.0) <= 0.2


def test_cli_restart(built, cuda_device, tmp_path):
    """A run that restarts (-r) from the checkpoint its loop wrote ends with
    the same grains, grain table and summary as the uninterrupted run.
    DataWriteStart 150 also sets the checkpoint frequency, as in the
    reference's parser (read_ctrl.c:594-600): checkpoints at steps 150 and
    300 of the 400."""
    deck = tmp_path / "small4_cp.in"
    deck.write_text((GOLDEN / "decks" / "small4.in").read_text() + "\nDataWriteStart 150\n")
    full = tmp_path / "full"
    full.mkdir()
    lines_full = run_cli(deck, full)
    assert (full / "cp_main.mms").exists()
    # a second directory gets the step-300 checkpoint, then restarts from it
    part = tmp_path / "part"
    part.mkdir()
    (part / "cp_main.mms").write_bytes((full / "cp_main.mms").read_bytes())
    lines_part = run_cli(deck, part, "-r", "1")
    assert any(b"restarting at timestep 300" in line for line in lines_part)
    assert summary(lines_part) == summary(lines_full)
    assert (part / "small4_grains.csv").read_bytes() == (full / "small4_grains.csv").read_bytes()
