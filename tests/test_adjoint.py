"""Frozen-CA adjoint through the C ABI (mms_adjoint_*).

The recording run must still be the reference's run bit for bit; the
frozen replay with the recorded parameters must reproduce it bit for bit;
the adjoint gradient must agree with central finite differences of the
replay (step 1e-4 relative) to 1e-4 relative, and the FP32 adjoint with the
FP64 one within the stated bound."""
from __future__ import annotations

import numpy as np
import pytest

import mumatscale_b200 as M
from conftest import golden, golden_deck
from digests import mismatches, state_digests

pytestmark = pytest.mark.gpu

NSTEPS, EVERY = 100, 40      # three checkpoint segments, the last one partial
FD_STEP = 1e-4               # central differences, relative step
FD_TOL = 1e-4                # adjoint vs finite differences, relative
F32_TOL = 2e-2               # FP32 adjoint vs FP64 adjoint, relative
PARAMS = ("Dliq", "part_coef", "gibbs")


def _target(name: str, prec: int) -> np.ndarray:
    """ce after NSTEPS of the deck with D_l x 1.2 and k x 0.9."""
    p = M.read_deck(golden_deck(name))
    p.Dliq *= 1.2
    p.part_coef *= 0.9
    with M.Domain(p, precision=prec) as d:
        d.step(NSTEPS)
        return d.download("ce")


@pytest.mark.parametrize("name", ["small4", "curv1"])
def test_recording_run_is_the_reference_run(built, cuda_device, name):
    rec = golden(name)
    want = rec["steps"][str(NSTEPS)] if str(NSTEPS) in rec["steps"] else None
    p = M.read_deck(golden_deck(name))
    with M.Domain(p, precision=M.PREC_F64) as dom:
        dom.adjoint_record(NSTEPS, EVERY)
        assert dom.timestep == NSTEPS
        if want is not None:
            assert mismatches(state_digests(dom), want["digest"]) == []
        with M.Domain(p, precision=M.PREC_F64) as ref:
            ref.step(NSTEPS)
            assert mismatches(state_digests(dom), state_digests(ref)) == []


@pytest.mark.parametrize("prec", [M.PREC_F64, M.PREC_F32])
def test_replay_reproduces_recorded_run(built, cuda_device, prec):
    p = M.read_deck(golden_deck("curv1"))
    with M.Domain(p, precision=prec) as dom:
        dom.adjoint_record(NSTEPS, EVERY)
        ce = dom.download("ce")
        # the final ce as target: the unperturbed replay must land on it exactly
        assert dom.adjoint_replay_loss(ce) == 0.0
        assert dom.adjoint_replay_loss(ce, (1.001, 1.0, 1.0)) > 0.0


def _fd(dom, target, which: int) -> float:
    up = [1.0, 1.0, 1.0]
    dn = [1.0, 1.0, 1.0]
    up[which] += FD_STEP
    dn[which] -= FD_STEP
    return (dom.adjoint_replay_loss(target, up) - dom.adjoint_replay_loss(target, dn)) / (2 * FD_STEP)


def test_fp64_gradient_vs_finite_differences(built, cuda_device):
    p = M.read_deck(golden_deck("curv1"))
    target = _target("curv1", M.PREC_F64)
    base = {"Dliq": p.Dliq, "part_coef": p.part_coef, "gibbs": p.gibbs_coef}
    with M.Domain(p, precision=M.PREC_F64) as dom:
        dom.adjoint_record(NSTEPS, EVERY)
        g = dom.adjoint_gradient(target)
        assert g["steps"] == NSTEPS
        assert g["loss"] > 0
        assert abs(g["loss"] - dom.adjoint_replay_loss(target)) <= 1e-13 * g["loss"]
        scale_grads = {k: g[k] * base[k] for k in PARAMS}   # dL/d(log theta)
        big = max(abs(v) for v in scale_grads.values())
        for i, k in enumerate(PARAMS):
            fd = _fd(dom, target, i)
            err = abs(scale_grads[k] - fd)
            # relative to the derivative itself, or to the largest one when
            # this parameter barely matters
            assert err <= FD_TOL * max(abs(fd), 1e-6 * big), (k, scale_grads[k], fd)
        assert abs(scale_grads["Dliq"]) > 0 and abs(scale_grads["part_coef"]) > 0


def test_fp32_adjoint_vs_fp64(built, cuda_device):
    p = M.read_deck(golden_deck("curv1"))
    target = _target("curv1", M.PREC_F64)
    base = {"Dliq": p.Dliq, "part_coef": p.part_coef, "gibbs": p.gibbs_coef}
    grads = {}
    for prec in (M.PREC_F64, M.PREC_F32):
        with M.Domain(p, precision=prec) as dom:
            dom.adjoint_record(NSTEPS, EVERY)
            grads[prec] = dom.adjoint_gradient(target)
    g64, g32 = grads[M.PREC_F64], grads[M.PREC_F32]
    assert abs(g32["loss"] / g64["loss"] - 1) < 1e-3
    big = max(abs(g64[k] * base[k]) for k in PARAMS)
    for k in PARAMS:
        a, b = g32[k] * base[k], g64[k] * base[k]
        assert abs(a - b) <= F32_TOL * max(abs(b), 1e-6 * big), (k, a, b)


def test_adjoint_requires_a_record(built, cuda_device):
    p = M.read_deck(golden_deck("small1"))
    with M.Domain(p) as dom:
        with pytest.raises(M.MmsError) as e:
            dom.adjoint_gradient(np.zeros(dom.num_cells()))
        assert e.value.status == 10  # MMS_ERR_STATE


def test_corrected_curvature_gibbs_gradient(built, cuda_device):
    """With the corrected curvature (mms_params.curvature_corrected) the
    Gibbs-Thomson term acts on generic interfaces, so dL/dGamma measures the
    physics rather than the reference's zero-curvature quirk
    (curvature.c:194, 203).  curv1 over 400 steps (checkpoints every 100):
    the adjoint agrees with central differences of the replay, and the
    Gibbs-Thomson derivative is larger than with the reference's formula."""
    steps, every = 400, 100
    base = None
    gib = {}
    for fixed in (0, 1):
        p = M.read_deck(golden_deck("curv1"))
        p.curvature_corrected = fixed
        pt = M.read_deck(golden_deck("curv1"))
        pt.curvature_corrected = fixed
        pt.Dliq *= 1.2
        pt.part_coef *= 0.9
        with M.Domain(pt, precision=M.PREC_F64) as d:
            d.step(steps)
            target = d.download("ce")
        base = {"Dliq": p.Dliq, "part_coef": p.part_coef, "gibbs": p.gibbs_coef}
        with M.Domain(p, precision=M.PREC_F64) as dom:
            dom.adjoint_record(steps, every)
            g = dom.adjoint_gradient(target)
            grads = {k: g[k] * base[k] for k in PARAMS}
            big = max(abs(v) for v in grads.values())
            if fixed:
                for i, k in enumerate(PARAMS):
                    fd = _fd(dom, target, i)
                    assert abs(grads[k] - fd) <= FD_TOL * max(abs(fd), 1e-6 * big), (k, grads[k], fd)
            gib[fixed] = abs(grads["gibbs"])
    assert gib[1] > 2 * gib[0], gib


def test_adjoint_cfg5_scale(built, cuda_device, tmp_path):
    """The calibration configuration at full size: the one-grain deck at
    128^3 cells with curvature, 2000 steps recorded with checkpoints every
    100; target ce from the same deck with D_l x 1.2 and k x 0.9.  The FP64
    adjoint agrees with central differences of the frozen replay (step 1e-4
    relative) to 1e-4 relative for D_l, k and the Gibbs-Thomson coefficient."""
    from mumatscale_b200 import workloads as W
    n, steps, every = 128, 2000, 100
    deck, cells, thr, rot = W.one_grain(n)
    f = tmp_path / "adj.in"
    f.write_text(deck)
    p = M.read_deck(f)
    pt = M.read_deck(f)
    pt.Dliq *= 1.2
    pt.part_coef *= 0.9
    with M.Domain(pt) as d:
        W.setup_one_grain(d, cells, thr, rot)
        d.step(steps)
        target = d.download("ce")
    base = {"Dliq": p.Dliq, "part_coef": p.part_coef, "gibbs": p.gibbs_coef}
    with M.Domain(p, precision=M.PREC_F64) as dom:
        W.setup_one_grain(dom, cells, thr, rot)
        dom.adjoint_record(steps, every)
        g = dom.adjoint_gradient(target)
        assert g["steps"] == steps and g["loss"] > 0
        grads = {k: g[k] * base[k] for k in PARAMS}
        big = max(abs(v) for v in grads.values())
        for i, k in enumerate(PARAMS):
            fd = _fd(dom, target, i)
            assert abs(grads[k] - fd) <= FD_TOL * max(abs(fd), 1e-6 * big), (k, grads[k], fd)
