"""Nucleation sites drawn on the device (mms_params.site_setup = 1): not the
reference's rand() sequence, so these tests check what the draw promises
against the host setup that replays the reference (init_sb_nucleation,
grain.c:930-1010): deterministic for a seed, site counts within binomial
bounds of the reference's exact counts, thresholds from the truncated
normal of genRandomThreshold (grain.c:140-154), deck-defined sites kept."""
from __future__ import annotations

import math
import tempfile
from pathlib import Path

import numpy as np
import pytest

import mumatscale_b200 as M
from conftest import ROOT, golden_deck

pytestmark = pytest.mark.gpu


def _bench_params(n: int, seed: int = 20261203) -> M.Params:
    import sys
    sys.path.insert(0, str(ROOT))
    import bench
    d = Path(tempfile.mkdtemp()) / "b.in"
    d.write_text(bench.deck_text(n=n, nsb=(2, 2, 2), seed=seed))
    return M.read_deck(d)


def _thresholds(p: M.Params) -> np.ndarray:
    with M.Domain(p) as dom:
        return dom.download("nuc_threshold")


def test_device_sites_statistics(built, cuda_device):
    """128^3, 2 x 2 x 2 ranks, 1e15 volume sites per m^3 (~16.8k) and the
    bench deck's surface sites: counts within 5 binomial sigma of the host
    setup's exact ones, volume thresholds' mean and sigma within 4 standard
    errors of N(2, 0.5)."""
    p = _bench_params(128)
    p.maxGrainDensity = 1e15
    host = _thresholds(p)
    import ctypes as C
    q = M.Params()
    C.pointer(q)[0] = p
    q.site_setup = 1
    dev = _thresholds(q)
    assert np.array_equal(dev, _thresholds(q)), "not deterministic for one seed"
    nh, nd = int(np.isfinite(host).sum()), int(np.isfinite(dev).sum())
    assert abs(nd - nh) <= 5 * math.sqrt(nh) + 5, (nd, nh)
    # interior (non-surface) sites are volume sites: N(2, 0.5) truncated at 6 sigma
    inner = dev[2:-2, 2:-2, 2:-2]
    t = inner[np.isfinite(inner)].astype(np.float64)
    assert len(t) > 10000
    se = p.gnGaussSigma / math.sqrt(len(t))
    assert abs(t.mean() - p.gnGaussCenter) < 4 * se
    assert abs(t.std() - p.gnGaussSigma) < 4 * se / math.sqrt(2) + 2e-3
    assert t.min() >= 1e-5 and np.abs(t - p.gnGaussCenter).max() <= 6 * p.gnGaussSigma + 1e-6
    # surface sites sit on the pad faces only: no site in the halo
    assert not np.isfinite(dev[0]).any() and not np.isfinite(dev[-1]).any()
    q.base_random_seed += 1
    assert not np.array_equal(_thresholds(q), dev)


def test_device_sites_keep_deck_sites_and_grow(built, cuda_device):
    p = M.read_deck(golden_deck("small4"))  # FixedNuc at threshold 0.5
    p.site_setup = 1
    with M.Domain(p) as dom:
        thr = dom.download("nuc_threshold")
        assert np.isclose(thr, 0.5).any()
        dom.step(200)
        assert dom.num_grains > 5


def test_device_sites_refused_on_slabs(built, cuda_device):
    p = M.read_deck(golden_deck("small4"))
    p.site_setup = 1
    with pytest.raises(M.MmsError):
        M.SlabDomain(p, 2, 0)
