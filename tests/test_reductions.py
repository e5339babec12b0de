"""Fraction-solid reductions after a step (computeFS, loop.c:173-183;
solid_volume, growth.c:541-566).

In mms_step_reduce the last step's stencil leaves one sum of the new
fraction solid per tile, which it folds (and mms_reduce after it reuses)
instead of reading the field again.  Every case compares with the sum of
the downloaded field (each value capped at 1, as reduce_fs does), including
the cases where the tile sums must NOT be used: a plain step since, fields
uploaded, a checkpoint loaded, the tile changed or tuned."""
from __future__ import annotations

import numpy as np
import pytest

import mumatscale_b200 as M
from conftest import golden_deck

pytestmark = pytest.mark.gpu

# plain FP64 sums in a different order from the field pass: a few ulps
REL = 1e-13


def _field_fraction(dom) -> float:
    fs = dom.download("fs")[1:-1, 1:-1, 1:-1]
    return float(np.sum(np.minimum(fs, 1.0), dtype=np.float64)) / fs.size


def _close(a: float, b: float) -> bool:
    return abs(a - b) <= REL * abs(b)


@pytest.mark.parametrize("prec", [M.PREC_F64, M.PREC_F32])
@pytest.mark.parametrize("tile", [(1, 0), (2, 8), (2, 16)])
def test_fraction_after_steps(built, cuda_device, prec, tile):
    p = M.read_deck(golden_deck("small4"))
    cells = p.gnsbx * p.gsdimx * p.gnsby * p.gsdimy * p.gnsbz * p.gsdimz
    with M.Domain(p, precision=prec) as dom:
        dom.set_stencil_tile(*tile)
        for n in (1, 37, 120, 8, 9):
            got = dom.step_reduce(n, "fs_fraction")
            want = _field_fraction(dom)
            assert 0 <= want < 1
            assert _close(got, want), (n, got, want)
            # mms_reduce reuses the tile sums of that step
            assert dom.reduce("fs_fraction") == got
            assert _close(dom.reduce("solid_volume"), want * cells * p.cellSize ** 3)
        assert want > 0
        # a plain step leaves no tile sums: the field pass
        dom.step(3)
        assert _close(dom.reduce("fs_fraction"), _field_fraction(dom))
        ce = dom.step_reduce(2, "ce_sum")
        assert abs(ce / float(np.sum(dom.download("ce")[1:-1, 1:-1, 1:-1])) - 1) < 1e-12
        assert _close(dom.reduce("fs_fraction"), _field_fraction(dom))


def test_fraction_follows_uploads_and_checkpoints(built, cuda_device, tmp_path):
    p = M.read_deck(golden_deck("small4"))
    with M.Domain(p) as dom:
        base = dom.step_reduce(80, "fs_fraction")
        ck = tmp_path / "s.ckpt"
        dom.checkpoint_save(str(ck))
        # an uploaded field replaces what the last step left
        fs = dom.download("fs")
        fs2 = fs.copy()
        fs2[1:-1, 1:-1, 1:-1] = np.where(fs2[1:-1, 1:-1, 1:-1] > 0, 1.0, 0.25)
        dom.upload("fs", fs2)
        got = dom.reduce("fs_fraction")
        assert _close(got, _field_fraction(dom)) and not _close(got, base)
        # a checkpoint of the earlier state brings its value back
        dom.checkpoint_load(str(ck))
        assert _close(dom.reduce("fs_fraction"), base)
        assert _close(dom.step_reduce(5, "fs_fraction"), _field_fraction(dom))


def test_fraction_after_tile_change_and_tuning(built, cuda_device):
    p = M.read_deck(golden_deck("small4"))
    with M.Domain(p) as dom:
        dom.set_stencil_tile(2, 8)
        dom.step_reduce(60, "fs_fraction")
        want = _field_fraction(dom)
        # another tile has another tile count: no step since, so the field pass
        dom.set_stencil_tile(1, 4)
        assert _close(dom.reduce("fs_fraction"), want)
        # tuning runs the stencil on shadow copies, which must not leak in
        dom.step_reduce(1, "fs_fraction")
        want = _field_fraction(dom)
        dom.autotune(2)
        assert _close(dom.reduce("fs_fraction"), want)
        assert _close(dom.step_reduce(3, "fs_fraction"), _field_fraction(dom))


def test_fraction_with_per_kernel_timing(built, cuda_device):
    """With per-kernel timing the step runs as separate launches, not as
    graphs; the tile sums are the same."""
    p = M.read_deck(golden_deck("small4"))
    with M.Domain(p) as a, M.Domain(p) as b:
        b.set_profiling(True)
        assert a.step_reduce(50, "fs_fraction") == b.step_reduce(50, "fs_fraction")
        assert _close(b.reduce("fs_fraction"), _field_fraction(b))


@pytest.mark.parametrize("prec", [M.PREC_F64, M.PREC_F32])
@pytest.mark.parametrize("sdimx", [5, 15, 33, 67])
def test_field_pass_ragged_rows(built, cuda_device, prec, sdimx):
    """The field pass over rows whose length is not a multiple of the
    16-byte vector: head and tail elements are each counted once."""
    p = M.read_deck(golden_deck("small4"))
    p.gsdimx = sdimx
    with M.Domain(p, precision=prec) as dom:
        dom.step(40)
        assert _close(dom.reduce("fs_fraction"), _field_fraction(dom))
        ce = dom.download("ce")[1:-1, 1:-1, 1:-1]
        assert abs(dom.reduce("ce_sum") / float(np.sum(ce)) - 1) < 1e-12
