"""Batched independent domains (mms_batch_*): every domain of a batch must
end in exactly the state it reaches when stepped alone."""
from __future__ import annotations

import pytest

import mumatscale_b200 as M
from mumatscale_b200 import workloads as W
from conftest import golden_deck
from digests import mismatches, state_digests


def _params(tmp_path, decks):
    out = []
    for i, d in enumerate(decks):
        f = tmp_path / f"d{i}.in"
        f.write_text(d)
        out.append(M.read_deck(f))
    return out


def test_ensemble_decks(built, tmp_path):
    decks = W.ensemble(64)
    assert len(decks) == 64
    ps = _params(tmp_path, decks[:8])
    for p in ps:
        assert {p.gsdimx, p.gsdimy, p.gsdimz} <= {32, 48, 64, 96, 128}
        assert 10 <= p.cool_rate <= 1000


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [M.PREC_F64, M.PREC_F32])
def test_batch_equals_domains_alone(built, cuda_device, tmp_path, prec):
    decks = W.ensemble(5, seed=5, edges=(20, 24, 36))
    ps = _params(tmp_path, decks) + [M.read_deck(golden_deck("small4")), M.read_deck(golden_deck("curv1"))]
    with M.Batch(ps, precision=prec) as b:
        b.step(60)
        b.autotune(reps=2)
        b.step(40)
        b.set_stencil_tile(2, 5)
        b.step(50)
        assert b.kernel_launches > 0
        for i, p in enumerate(ps):
            with M.Domain(p, precision=prec) as d:
                d.step(150)
                got = b.domains[i]
                assert got.timestep == 150
                assert got.num_grains == d.num_grains
                assert mismatches(state_digests(got), state_digests(d)) == [], i
