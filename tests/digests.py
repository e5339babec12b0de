"""Field digests in the layout of tests/golden/*.json (test infrastructure)."""
from __future__ import annotations

import hashlib

import numpy as np


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def state_digests(dom) -> dict:
    """dom: a mumatscale_b200.Domain or a tests._oracle.Oracle."""
    out = {f: digest(dom.download(f)) for f in ("ce", "cl", "fs", "gr", "dc", "nuc_threshold", "d")}
    grains = dom.grains()
    rot = np.array([np.array(g.rotmat).reshape(9) for g in grains[1:]], dtype="<f8").reshape(-1, 9)
    out["grain_rotmat"] = digest(rot)
    out["grain_ts"] = digest(np.array([g.nuc_timestep for g in grains[1:]], dtype="<u8"))
    return out


def mismatches(got: dict, want: dict) -> list[str]:
    return [k for k in want if got.get(k) != want[k]]
