"""ParaView output in the io_vtk.c layout (host side; no GPU)."""
from __future__ import annotations

import xml.etree.ElementTree as ET

import numpy as np
import pytest

import mumatscale_b200 as M
from conftest import golden_deck


def _arr(piece, name):
    for da in piece.iter("DataArray"):
        if da.get("Name") == name:
            return da
    raise KeyError(name)


def test_vtk_layout_matches_reference_writer(built, tmp_path):
    p = M.read_deck(golden_deck("small4"))          # 2 x 2 x 1 subblocks
    gx, gy, gz = p.grid
    rng = np.random.default_rng(3)
    T = rng.normal(1600, 5, (gz + 2, gy + 2, gx + 2))
    gr = rng.integers(0, 50, (gz + 2, gy + 2, gx + 2)).astype(np.int32)
    base = str(tmp_path / "out")
    M.write_vtk_arrays(p, base, 42, T, gr)
    pv = ET.parse(base + "_42.pvtu").getroot()
    pieces = [e.get("Source") for e in pv.iter("Piece")]
    nsub = p.gnsbx * p.gnsby * p.gnsbz
    assert pieces == [f"{base}_{s:04d}/42.vtu" for s in range(nsub)]
    dx, dy, dz = p.gsdimx, p.gsdimy, p.gsdimz
    for s in range(nsub):
        sx, sy, sz = s % p.gnsbx, (s // p.gnsbx) % p.gnsby, s // (p.gnsbx * p.gnsby)
        root = ET.parse(f"{base}_{s:04d}/42.vtu").getroot()
        piece = next(root.iter("Piece"))
        assert int(piece.get("NumberOfCells")) == dx * dy * dz
        assert int(piece.get("NumberOfPoints")) == (dx + 1) * (dy + 1) * (dz + 1)
        temp = np.array(_arr(piece, "Temperature").text.split(), dtype=float)
        grain = np.array(_arr(piece, "Grain").text.split(), dtype=int)
        # writeDataArrayFloat/Int32 (io_vtk.c:95-200): x outer, z inner, interior cells
        sub = (slice(sz * dz + 1, sz * dz + dz + 1), slice(sy * dy + 1, sy * dy + dy + 1),
               slice(sx * dx + 1, sx * dx + dx + 1))
        want_t = np.transpose(T[sub], (2, 1, 0)).ravel()
        assert np.allclose(temp, want_t, rtol=0, atol=5e-7)          # "%lf"
        assert np.array_equal(grain, np.transpose(gr[sub], (2, 1, 0)).ravel())
        types = np.array(_arr(piece, "types").text.split(), dtype=int)
        assert (types == 11).all() and len(types) == dx * dy * dz
        offs = np.array(_arr(piece, "offsets").text.split(), dtype=int)
        assert offs[0] == 8 and offs[-1] == 8 * dx * dy * dz
        conn = np.array(_arr(piece, "connectivity").text.split(), dtype=int).reshape(-1, 8)
        row, plane = dz + 1, (dy + 1) * (dz + 1)
        assert list(conn[0]) == [0, 1, row, row + 1, plane, plane + 1, plane + row, plane + row + 1]
        pts = np.array(next(piece.iter("Points")).find("DataArray").text.split(), dtype=float).reshape(-1, 3)
        x0 = p.origin_offset[0] + (sx * dx + 0.5) * p.cellSize
        assert abs(pts[0, 0] - x0) <= 1e-6 * abs(x0) + 1e-12


@pytest.mark.gpu
def test_vtk_from_device(built, cuda_device, tmp_path):
    p = M.read_deck(golden_deck("small1"))
    with M.Domain(p) as dom:
        dom.step(100)
        base = str(tmp_path / "dev")
        dom.write_vtk(base)
        piece = next(ET.parse(f"{base}_0000/100.vtu").getroot().iter("Piece"))
        grain = np.array(_arr(piece, "Grain").text.split(), dtype=int)
        gr = dom.download("gr")[1:-1, 1:-1, 1:-1]
        assert np.array_equal(grain, np.transpose(gr, (2, 1, 0)).ravel())
