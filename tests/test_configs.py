"""The synthetic workloads of mumatscale_b200.workloads run through the C ABI
against the oracle (bit-exact in the FP64 plain form)."""
from __future__ import annotations

import pytest

import mumatscale_b200 as M
from mumatscale_b200 import workloads as W
from digests import mismatches, state_digests


def test_one_grain_deck_parses(built, tmp_path):
    deck, cells, thr, rot = W.one_grain(64)
    f = tmp_path / "og.in"
    f.write_text(deck)
    p = M.read_deck(f)
    assert (p.gsdimx, p.gsdimy, p.gsdimz) == (64, 64, 64)
    assert abs(p.Dliq * p.ts_delt / p.cellSize ** 2 - W.FOURIER) < 1e-12
    assert 3 * W.FOURIER < W.K_PART        # the stability bound the decks keep
    assert cells.shape == (1, 3) and rot.shape == (1, 9)


@pytest.mark.gpu
def test_one_grain_64_bit_exact_vs_oracle(built, cuda_device, tmp_path):
    """64^3 one-grain deck without curvature, 2000 steps: bit-identical state."""
    from _oracle import Oracle
    deck, cells, thr, rot = W.one_grain(64, tip_curv=0)
    f = tmp_path / "og.in"
    f.write_text(deck)
    p = M.read_deck(f)
    o = Oracle(p)
    W.setup_one_grain(o, cells, thr, rot)
    with M.Domain(p, precision=M.PREC_F64) as dom:
        W.setup_one_grain(dom, cells, thr, rot)
        for s in (1, 500, 2000):
            o.step(s - o.timestep)
            dom.step(s - dom.timestep)
            assert mismatches(state_digests(dom), state_digests(o)) == [], s
        assert dom.num_grains == 2
        assert 0 < dom.reduce("fs_fraction") < 1


@pytest.mark.gpu
def test_one_grain_64_curvature_vs_oracle(built, cuda_device, tmp_path):
    """With TipCurvature the reference divides by glibc's pow(x, 1.5), which
    misrounds a small fraction of inputs (about 1 in 1000 in a uniform
    sample); the device computes the correctly rounded value.  Bounds after
    2000 steps: ce relative L2 error < 1e-2, grain-id mismatch < 1e-3 of the
    cells, the same grain count."""
    import numpy as np
    from _oracle import Oracle
    deck, cells, thr, rot = W.one_grain(64, tip_curv=1)
    f = tmp_path / "og.in"
    f.write_text(deck)
    p = M.read_deck(f)
    o = Oracle(p)
    W.setup_one_grain(o, cells, thr, rot)
    with M.Domain(p, precision=M.PREC_F64) as dom:
        W.setup_one_grain(dom, cells, thr, rot)
        o.step(2000)
        dom.step(2000)
        ce, ce0 = dom.download("ce"), o.download("ce")
        rel = float(np.linalg.norm(ce - ce0) / np.linalg.norm(ce0))
        mism = float((dom.download("gr") != o.download("gr")).mean())
        assert rel < 1e-2 and mism < 1e-3, (rel, mism)
        assert dom.num_grains == o.num_grains


@pytest.mark.gpu
def test_prefilled_grains_bit_exact_vs_oracle(built, cuda_device):
    """A substrate of injected grains (mms_set_grains + field uploads) grows
    like the oracle's, bit for bit."""
    import numpy as np
    from _oracle import Oracle
    from conftest import golden_deck
    p = M.read_deck(golden_deck("small1"))
    o = Oracle(p)
    rng = np.random.default_rng(7)
    with M.Domain(p, precision=M.PREC_F64) as dom:
        gr = dom.download("gr")
        fs = dom.download("fs")
        cl = dom.download("cl")
        ce = dom.download("ce")
        nz, ny, nx = gr.shape
        # three columnar grains in the bottom four planes
        cols = rng.integers(1, 4, size=(ny, nx))
        gr[1:5, 1:-1, 1:-1] = cols[None, 1:-1, 1:-1]
        fs[1:5, 1:-1, 1:-1] = 1.0
        rot = np.stack([W.quat_to_rotmat(q).ravel() for q in W.random_quaternions(rng, 3)])
        for d in (dom, o):
            d.set_grains(rot)
            d.upload("gr", gr)
            d.upload("fs", fs)
            d.upload("cl", cl)
            d.upload("ce", ce)
        assert dom.num_grains == 4 and o.num_grains == 4
        for s in (50, 200):
            o.step(s - o.timestep)
            dom.step(s - dom.timestep)
            assert mismatches(state_digests(dom), state_digests(o)) == [], s
        assert dom.num_grains > 4


@pytest.mark.gpu
@pytest.mark.parametrize("sb", [(32, 12, 10), (64, 6, 5)])
def test_word_aligned_subblocks_bit_exact_vs_oracle(built, cuda_device, sb):
    """small4's physics with subblock rows a multiple of 32 cells (the
    interface list then reads whole bitmask words per 32-cell piece) over
    2 x 1 x 2 emulated ranks: bit-identical state to the oracle."""
    from _oracle import Oracle
    from conftest import golden_deck
    p = M.read_deck(golden_deck("small4"))
    p.gsdimx, p.gsdimy, p.gsdimz = sb
    o = Oracle(p)
    with M.Domain(p, precision=M.PREC_F64) as dom:
        for s in (1, 100, 250):
            o.step(s - o.timestep)
            dom.step(s - dom.timestep)
            assert dom.num_grains == o.num_grains
            assert mismatches(state_digests(dom), state_digests(o)) == [], s
        assert dom.num_grains > 10


@pytest.mark.gpu
def test_corrected_curvature_vs_oracle(built, cuda_device):
    """mms_params.curvature_corrected = 1: the three quirks of sb_curvature
    fixed (curvature.c:176, 194, 203) on both sides.  On the curvature golden
    deck the device's curvature field equals the oracle's (to the last bits
    glibc's pow(x, 1.5) and the device's correctly rounded x^1.5 allow); it
    is non-zero on over a thousand interface cells at step 400, where the
    reference's own formula gives none (it is 0 unless a normal component
    is exactly 0)."""
    import numpy as np
    from _oracle import Oracle
    from conftest import golden_deck
    counts = {}
    for fixed in (0, 1):
        p = M.read_deck(golden_deck("curv1"))
        p.curvature_corrected = fixed
        o = Oracle(p, curvature=True)
        with M.Domain(p, precision=M.PREC_F64) as dom:
            for s in (200, 400):
                o.step(s - o.timestep)
                dom.step(s - dom.timestep)
                c, c0 = dom.download("curv"), o.download("curv")
                assert np.array_equal(c != 0, c0 != 0), (fixed, s)
                assert np.allclose(c, c0, rtol=1e-9, atol=0), (fixed, s)
            counts[fixed] = int((c0 != 0).sum())
    assert counts[0] == 0 and counts[1] > 1000, counts
