"""The reference's own regression answers, reproduced by the CUDA path.

tests/testOneGrain.py:25-39 (one_grain.in, 6 ranks): 1 grain, average
0.000737875 mm^3 +- 1e-6.  tests/testMultiGrains.py:25-37 (ca6mpi.in, 6
ranks): 336 grains, average 7.14e-5 mm^3 +- 1e-6.  The decks are restated
under tests/golden/decks with the reference's values (same keywords and
numbers), so this file does not read the reference tree."""
from __future__ import annotations

import pytest

import mumatscale_b200 as M
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def run_deck(name: str, precision: int = M.PREC_F64) -> M.GrainSummary:
    p = M.read_deck(GOLDEN / "decks" / f"{name}.in")
    with M.Domain(p, precision=precision) as dom:
        dom.run(verbose=0)
        return dom.grain_summary()


def test_one_grain(built, cuda_device):
    s = run_deck("one_grain")
    assert s.num_grains == 1
    assert abs(s.avg_mm3 - 0.000737875) <= 1e-6


def test_multi_grains(built, cuda_device):
    s = run_deck("ca6mpi")
    assert s.num_grains == 336
    assert abs(s.avg_mm3 - 7.14e-5) <= 1e-6
