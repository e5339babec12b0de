"""Pins the CPU oracle to the reference: every field of the oracle's state must
hash identically to the reference's own dumps (tests/golden/*.json, made by
tests/golden/make_golden.py from the unmodified reference sources).  CPU only."""
from __future__ import annotations

import pytest

import mumatscale_b200 as M
from conftest import GOLDEN_DECKS, golden, golden_deck, setup_golden_substrate
from digests import digest, mismatches, state_digests

# recorded steps checked on the CPU, where the whole record would take long:
# amsub4's laser turns on at step 8 (400 exponentials per cell and step from
# then on in the CPU oracle, as in the reference)
MAX_STEP = {"amsub4": 20}


@pytest.mark.parametrize("name", GOLDEN_DECKS)
def test_oracle_matches_reference_dumps(built, name):
    from _oracle import Oracle
    rec = golden(name)
    p = M.read_deck(golden_deck(name))
    o = Oracle(p, curvature=bool(rec["env"].get("MMSREF_CURV")))
    assert digest(o.download("nuc_threshold")) == rec["setup"]["nuc_threshold"]
    setup_golden_substrate(o, name)
    last = 0
    for s, want in rec["steps"].items():
        s = int(s)
        if s > MAX_STEP.get(name, 1 << 30):
            break
        o.step(s - last)
        last = s
        assert o.timestep == s
        assert o.num_grains == want["num_grains"]
        bad = mismatches(state_digests(o), want["digest"])
        assert not bad, f"{name} step {s}: fields differ from the reference: {bad}"
    if "error_at_step" in rec:
        with pytest.raises(RuntimeError, match="status 6"):
            o.step(rec["error_at_step"] - last)


def test_oracle_rand_matches_libc(built):
    """The per-rank streams replay glibc rand() (ca_main.c:215 srand)."""
    import ctypes
    from _oracle import rand_sequence
    libc = ctypes.CDLL("libc.so.6")
    for seed in (1, 7, 3823798713):
        libc.srand(ctypes.c_uint(seed))
        want = [libc.rand() for _ in range(500)]
        assert rand_sequence(seed, 500).tolist() == want
