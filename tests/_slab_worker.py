"""One rank of a slab-split run (test infrastructure): launched by
tests/test_slabs.py as a process per slab; steps its slab with
mumatscale_b200.slabs.DistributedSlab over a gloo group (host transport) or
an NCCL group (the library's own NCCL step loop) and saves its fields and
grain records to <out>/slab<rank>.npz."""
from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--deck", required=True)
    ap.add_argument("--nsbz", type=int, required=True)
    ap.add_argument("--sdimz", type=int, required=True)
    ap.add_argument("--steps", type=int, required=True)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--out", required=True)
    ap.add_argument("--backend", default="gloo", choices=["gloo", "nccl"])
    a = ap.parse_args()
    import numpy as np
    import torch.distributed as dist

    import mumatscale_b200 as M
    from mumatscale_b200.slabs import DistributedSlab
    if a.backend == "nccl":
        import torch
        torch.cuda.set_device(0)
    dist.init_process_group(a.backend, init_method="env://",
                            timeout=__import__("datetime").timedelta(seconds=120))
    p = M.read_deck(a.deck)
    p.gnsbz, p.gsdimz = a.nsbz, a.sdimz
    s = DistributedSlab(p, precision=a.precision, device=0)
    s.step(a.steps)
    d = s.dom
    out = {f: d.download(f) for f in ("ce", "cl", "fs", "gr", "dc")}
    g = d.grains()
    out["rot"] = np.array([np.array(x.rotmat).reshape(9) for x in g]).reshape(-1, 9)
    out["ang"] = np.array([list(x.rotang) for x in g]).reshape(-1, 3)
    out["nuc"] = np.array([[x.nuc_x, x.nuc_y, x.nuc_z, x.nuc_threshold, float(x.nuc_timestep)] for x in g])
    out["z_begin"] = np.array(d.layout.z_begin)
    out["timestep"] = np.array(s.timestep)
    out["red"] = np.array([s.reduce(w) for w in ("fs_fraction", "solid_volume", "ce_sum")])
    np.savez(os.path.join(a.out, f"slab{dist.get_rank()}.npz"), **out)
    s.close()
    dist.barrier()
    dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
