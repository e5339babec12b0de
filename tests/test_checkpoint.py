"""Raw checkpoint/restart (mms_checkpoint_save / mms_checkpoint_load): a
context loaded from a checkpoint continues bit for bit like the saved one."""
from __future__ import annotations

import numpy as np
import pytest

import mumatscale_b200 as M
from mumatscale_b200 import workloads as W
from conftest import golden_deck
from digests import mismatches, state_digests

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,prec", [("small4", M.PREC_F64), ("nucvol1", M.PREC_F64), ("curv1", M.PREC_F64),
                                       ("small4", M.PREC_F32)])
def test_restart_continues_exactly(built, cuda_device, tmp_path, name, prec):
    p = M.read_deck(golden_deck(name))
    ck = tmp_path / "state.ckpt"
    with M.Domain(p, precision=prec) as a:
        a.step(60)
        a.checkpoint_save(ck)
        a.step(100)
        want = state_digests(a)
        ng = a.num_grains
        ga = a.grains()
    with M.Domain(p, precision=prec) as b:
        b.checkpoint_load(ck)
        assert b.timestep == 60
        b.step(100)
        assert b.num_grains == ng
        assert mismatches(state_digests(b), want) == []
        gb = b.grains()
        for x, y in zip(ga[1:], gb[1:]):
            assert (x.nuc_x, x.nuc_y, x.nuc_z, x.nuc_timestep) == (y.nuc_x, y.nuc_y, y.nuc_z, y.nuc_timestep)


def test_restart_with_prefilled_grains(built, cuda_device, tmp_path):
    p = M.read_deck(golden_deck("small1"))
    ck = tmp_path / "sub.ckpt"
    with M.Domain(p) as a:
        W.setup_substrate(a, 3, p.cellSize, mean_width=3 * p.cellSize, seed=5)
        a.step(40)
        a.checkpoint_save(ck)
        a.step(60)
        want = state_digests(a)
    with M.Domain(p) as b:
        b.checkpoint_load(ck)
        b.step(60)
        assert mismatches(state_digests(b), want) == []
        rot = np.array(b.grains()[1].rotmat)
        assert abs(abs(np.linalg.det(rot)) - 1) < 1e-12


def test_checkpoint_of_another_deck_is_refused(built, cuda_device, tmp_path):
    ck = tmp_path / "a.ckpt"
    with M.Domain(M.read_deck(golden_deck("small1"))) as a:
        a.step(5)
        a.checkpoint_save(ck)
    with M.Domain(M.read_deck(golden_deck("small4"))) as b:
        with pytest.raises(M.MmsError) as e:
            b.checkpoint_load(ck)
        assert e.value.status == 1
