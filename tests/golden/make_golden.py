"""Generates the golden fixtures under tests/golden/ from the muMatScale
reference itself.

For every deck in tests/golden/decks/ (see DECKS below) this runs the
unmodified reference, compiled from its own sources by oracle/Makefile
(oracle/_ref/mmsref, with the project's MPI shim so NSubblocks > 1 runs as
that many processes), dumps its fields after the listed steps through the
link-time hooks in oracle/ref_shim/ref_hooks.c, and records a SHA-256 of
every field (the global halo'd array in the reference's index order) plus
a few readable summaries.  tests/test_oracle_golden.py recomputes the same
digests from the CPU oracle; the GPU tests compare the CUDA path with the
oracle.

Run in the build container (needs the reference sources):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(HERE))
from refdump import load_step  # noqa: E402

sys.path.insert(0, str(ROOT))
import mumatscale_b200 as M  # noqa: E402  (deck parser only)

REF = ROOT / "oracle" / "_ref" / "mmsref"

# deck -> (steps to dump, extra environment)
DECKS = {
    "small1": ([1, 50, 100, 200, 300, 400], {}),
    "small4": ([1, 50, 100, 200, 300, 400], {}),
    "cap1": ([50, 100], {"expect_error": "1"}),
    "curv1": ([100, 200, 300, 400], {"MMSREF_CURV": "1"}),
    "grad1": ([50, 150, 250, 350], {}),
    "nucvol1": ([1, 100, 200, 300], {}),
    "am1": ([1, 100, 110, 120, 130], {}),
    # reduced cfg3-shaped deck: AM source, columnar substrate of planes 1..24
    # (mean width 20 um, seed 11, injected on both sides), bulk sites, 4 ranks
    "amsub4": ([1, 7, 8, 15, 20, 30, 50, 100, 200, 300], {"substrate": "24,20e-6,11"}),
}

FIELDS = ("ce", "cl", "fs", "gr", "dc", "nuc_threshold", "d")


def digest(arr: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(arr).tobytes()).hexdigest()


def field_digests(st: dict) -> dict:
    out = {}
    for f in FIELDS:
        a = st[f]
        if f == "d":
            # d is defined where grow_octahedra computed it this step: cells
            # solid before capture (ogr > 0); elsewhere it holds stale values
            a = np.where(st["ogr"] > 0, a, 0.0)
        out[f] = digest(a)
    rot = np.array([g["rotmat"] for g in st["grains"]], dtype="<f8").reshape(-1, 9)
    out["grain_rotmat"] = digest(rot[1:])
    out["grain_ts"] = digest(np.array([g["ts"] for g in st["grains"]], dtype="<u8")[1:])
    return out


def deck_nsb(path: Path) -> tuple[int, int, int]:
    for line in path.read_text().splitlines():
        w = line.split()
        if w and w[0].lower() == "nsubblocks":
            return int(w[1]), int(w[2]), int(w[3])
    return 1, 1, 1


def main() -> None:
    if not REF.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    only = sys.argv[1:]
    for name, (steps, env_extra) in DECKS.items():
        if only and name not in only:
            continue
        deck = HERE / "decks" / f"{name}.in"
        nsb = deck_nsb(deck)
        env_extra = dict(env_extra)
        expect_error = bool(env_extra.pop("expect_error", ""))
        substrate = env_extra.pop("substrate", None)
        with tempfile.TemporaryDirectory() as td:
            env = dict(os.environ, MMSREF_NP=str(nsb[0] * nsb[1] * nsb[2]), MMSREF_DUMP_DIR=td,
                       MMSREF_DUMP_STEPS=",".join(map(str, steps)), MMSREF_DUMP_SETUP="1", **env_extra)
            sub_rec = None
            if substrate:
                from mumatscale_b200 import workloads as W
                top, width, seed = substrate.split(",")
                p = M.read_deck(deck)
                gx, gy = p.gnsbx * p.gsdimx, p.gnsby * p.gsdimy
                cols, rot = W.columnar_columns(gx, gy, p.cellSize, float(width), int(seed))
                W.write_substrate_file(Path(td) / "substrate.bin", cols, rot, int(top))
                env["MMSREF_INJECT_SUBSTRATE"] = str(Path(td) / "substrate.bin")
                sub_rec = {"top_plane": int(top), "mean_width": float(width), "seed": int(seed),
                           "cols": digest(cols.astype("<i4")), "rotmat": digest(rot.astype("<f8"))}
            if expect_error:
                env["MMSREF_DUMP_EVERY"] = "1"
            r = subprocess.run([str(REF), "-c", str(deck)], cwd=td, env=env, capture_output=True, text=True)
            if (r.returncode != 0) != expect_error:
                raise SystemExit(f"{name}: unexpected reference exit {r.returncode}\n{r.stdout}\n{r.stderr}")
            summary = [l for l in r.stdout.splitlines() if "Average" in l]
            rec = {"deck": f"decks/{name}.in", "nsubblocks": nsb, "env": env_extra,
                   "summary_line": summary[-1] if summary else None, "steps": {}}
            if sub_rec:
                rec["substrate"] = sub_rec
            if expect_error:
                done = [int(f.stem.split("_s")[1]) for f in Path(td).glob("r0_s[0-9]*.bin")]
                rec["error_at_step"] = max(done) + 1
                rec["error"] = [l for l in r.stderr.splitlines() if "ERROR" in l][-1].split("] ", 1)[-1]
                steps = sorted({s for s in steps if s < rec["error_at_step"]} | {rec["error_at_step"] - 1})
            st = load_step(td, "setup", nsb)
            rec["setup"] = {"nuc_threshold": digest(st["nuc_threshold"]),
                            "n_sites": int(np.isfinite(st["nuc_threshold"]).sum())}
            for s in steps:
                st = load_step(td, f"s{s}", nsb)
                gr = st["gr"]
                rec["steps"][str(s)] = {
                    "num_grains": st["num_grains"],
                    "solid_cells": int((gr[1:-1, 1:-1, 1:-1] > 0).sum()),
                    "ce_sum": float(st["ce"][1:-1, 1:-1, 1:-1].sum()),
                    "fs_sum": float(st["fs"][1:-1, 1:-1, 1:-1].sum()),
                    "digest": field_digests(st),
                }
        (HERE / f"{name}.json").write_text(json.dumps(rec, indent=1) + "\n")
        print(name, rec["summary_line"])


def vtk_record() -> None:
    """SHA-256 of every file the reference's VTK writer (io_vtk.c, its
    default zlib + base64 encoding) produces for small4 with DataFormat VTK
    and DataWriteFreq 200: steps 0, 200, 400 and the final 401 -> vtk_small4.json."""
    deck_src = HERE / "decks" / "small4.in"
    with tempfile.TemporaryDirectory() as td:
        deck = Path(td) / "small4_vtk.in"
        deck.write_text(deck_src.read_text() + "\nDataFormat VTK\nDataWriteFreq 200\n")
        nsb = deck_nsb(deck_src)
        env = dict(os.environ, MMSREF_NP=str(nsb[0] * nsb[1] * nsb[2]))
        r = subprocess.run([str(REF), "-c", str(deck)], cwd=td, env=env, capture_output=True, text=True)
        if r.returncode != 0:
            raise SystemExit(f"vtk: reference exited {r.returncode}\n{r.stderr}")
        files = {}
        for f in sorted(Path(td).rglob("*")):
            if f.is_file() and f.suffix in (".vtu", ".pvtu"):
                files[str(f.relative_to(td))] = hashlib.sha256(f.read_bytes()).hexdigest()
    rec = {"deck": "decks/small4.in", "extra": ["DataFormat VTK", "DataWriteFreq 200"], "files": files}
    (HERE / "vtk_small4.json").write_text(json.dumps(rec, indent=1) + "\n")
    print("vtk", len(files), "files")


if __name__ == "__main__":
    if sys.argv[1:] == ["vtk"]:
        vtk_record()
    else:
        main()
