"""Reader for the field dumps written by oracle/ref_shim/ref_hooks.c (the
reference's own state after a step), and assembly of per-rank dumps into
one global halo'd array.  Test infrastructure."""
from __future__ import annotations

from pathlib import Path

import numpy as np

GRAIN_DTYPE = np.dtype([("nuc", "<f8", 3), ("ts", "<u8"), ("thr", "<f8"),
                        ("rotmat", "<f8", 9), ("rotang", "<f8", 3)])


def read_dump(path: str | Path) -> dict:
    raw = Path(path).read_bytes()
    if raw[:8] != b"MMSDUMP1":
        raise ValueError(f"{path}: not a dump")
    hdr = np.frombuffer(raw, dtype="<i8", count=12, offset=8)
    (rank, nproc, sbx, sby, sbz, dx, dy, dz, ts, ngr, maxg, gindex) = (int(v) for v in hdr)
    n = (dx + 2) * (dy + 2) * (dz + 2)
    off = 8 + 12 * 8
    out = dict(rank=rank, nproc=nproc, coords=(sbx, sby, sbz), dims=(dx, dy, dz), timestep=ts,
               num_grains=ngr, max_grains=maxg, gindex=gindex)
    shape = (dz + 2, dy + 2, dx + 2)

    def take(dtype, count, shp=None):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a.reshape(shp) if shp else a

    out["ce"] = take("<f8", n, shape)
    out["cl"] = take("<f8", n, shape)
    out["fs"] = take("<f8", n, shape)
    out["d"] = take("<f8", n, shape)
    out["dc"] = take("<f8", 3 * n, shape + (3,))
    out["gr"] = take("<i4", n, shape)
    out["nuc_threshold"] = take("<f4", n, shape)
    out["temperature"] = take("<f8", n, shape)
    out["ogr"] = take("<i4", n, shape)
    out["grains"] = np.frombuffer(raw, dtype=GRAIN_DTYPE, count=ngr, offset=off)
    return out


def assemble(dumps: list[dict], nsb: tuple[int, int, int]) -> dict:
    """Stitch per-rank dumps (interior cells) into global halo'd arrays.

    Halo cells of the global array are taken from the ranks that own the
    corresponding boundary face."""
    d0 = dumps[0]
    sx, sy, sz = d0["dims"]
    gx, gy, gz = sx * nsb[0], sy * nsb[1], sz * nsb[2]
    out = {k: d0[k] for k in ("timestep", "num_grains", "grains")}
    for name in ("ce", "cl", "fs", "d", "dc", "gr", "nuc_threshold", "temperature", "ogr"):
        a0 = d0[name]
        shape = (gz + 2, gy + 2, gx + 2) + a0.shape[3:]
        g = np.zeros(shape, dtype=a0.dtype)
        for dd in dumps:
            cx, cy, cz = dd["coords"]
            a = dd[name]
            # every rank writes its full halo'd block; interior of later ranks
            # overwrites halos of earlier ones, so write halos first
            z0, y0, x0 = cz * sz, cy * sy, cx * sx
            g[z0:z0 + sz + 2, y0:y0 + sy + 2, x0:x0 + sx + 2] = np.where(
                np.zeros(a.shape, dtype=bool), 0, a)
        for dd in dumps:
            cx, cy, cz = dd["coords"]
            a = dd[name]
            z0, y0, x0 = cz * sz, cy * sy, cx * sx
            g[z0 + 1:z0 + sz + 1, y0 + 1:y0 + sy + 1, x0 + 1:x0 + sx + 1] = a[1:-1, 1:-1, 1:-1]
        out[name] = g
    return out


def load_step(dump_dir: str | Path, tag: str, nsb: tuple[int, int, int]) -> dict:
    nr = nsb[0] * nsb[1] * nsb[2]
    dumps = [read_dump(Path(dump_dir) / f"r{r}_{tag}.bin") for r in range(nr)]
    return assemble(dumps, nsb)
