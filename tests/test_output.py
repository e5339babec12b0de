"""ParaView (io_vtk.c) and XDMF (io_xdmf.c) output in the reference's layouts."""
from __future__ import annotations

import xml.etree.ElementTree as ET

import numpy as np
import pytest

from pathlib import Path

import mumatscale_b200 as M
from conftest import golden_deck
from digests import mismatches, state_digests


def _arr(piece, name):
    for da in piece.iter("DataArray"):
        if da.get("Name") == name:
            return da
    raise KeyError(name)


_DT = {"Float64": "<f8", "Int32": "<i4", "UInt8": "u1"}


def _decode(da) -> np.ndarray:
    """A DataArray in VTK's zlib block encoding (vtkZLibDataCompressor, 32-bit
    header): base64 header {blocks, block size, last size, compressed sizes},
    then the base64 of the concatenated zlib blocks."""
    import base64
    import zlib
    text = "".join(da.text.split())
    nb = int(np.frombuffer(base64.b64decode(text[:8])[:4], "<u4")[0])
    hlen = (3 + nb) * 4
    henc = (hlen + 2) // 3 * 4
    hdr = np.frombuffer(base64.b64decode(text[:henc]), "<u4")
    data = base64.b64decode(text[henc:])
    out, off = [], 0
    for c in hdr[3:3 + nb]:
        out.append(zlib.decompress(data[off:off + c]))
        off += int(c)
    return np.frombuffer(b"".join(out), _DT[da.get("type")])


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
        assert root.get("compressor") == "vtkZLibDataCompressor"
        piece = next(root.iter("Piece"))
        assert int(piece.get("NumberOfCells")) == dx * dy * dz
        assert int(piece.get("NumberOfPoints")) == (dx + 1) * (dy + 1) * (dz + 1)
        temp = _decode(_arr(piece, "Temperature"))
        grain = _decode(_arr(piece, "Grain"))
        # writeDataArrayFloat/Int32 (io_vtk.c:95-200): x outer, z inner, interior cells
        sub = (slice(sz * dz + 1, sz * dz + dz + 1), slice(sy * dy + 1, sy * dy + dy + 1),
               slice(sx * dx + 1, sx * dx + dx + 1))
        assert np.array_equal(temp, np.transpose(T[sub], (2, 1, 0)).ravel())   # raw doubles
        assert np.array_equal(grain, np.transpose(gr[sub], (2, 1, 0)).ravel())
        types = _decode(_arr(piece, "types"))
        assert (types == 11).all() and len(types) == dx * dy * dz
        offs = _decode(_arr(piece, "offsets"))
        assert offs[0] == 8 and offs[-1] == 8 * dx * dy * dz
        conn = _decode(_arr(piece, "connectivity")).reshape(-1, 8)
        row, plane = dz + 1, (dy + 1) * (dz + 1)
        assert list(conn[0]) == [0, 1, row, row + 1, plane, plane + 1, plane + row, plane + row + 1]
        pts = _decode(next(piece.iter("Points")).find("DataArray")).reshape(-1, 3)
        assert pts[0, 0] == p.origin_offset[0] + (sx * dx + 0.5) * p.cellSize


def _vtk_deck(tmp_path: Path) -> Path:
    from conftest import golden
    rec = golden("vtk_small4")
    deck = tmp_path / "small4_vtk.in"
    deck.write_text(golden_deck("small4").read_text() + "\n" + "\n".join(rec["extra"]) + "\n")
    return deck


def test_vtk_bytes_match_reference_files(built, tmp_path):
    """The writer fed with the CPU oracle's fields (pinned to the reference)
    produces the reference's own VTK files byte for byte: small4 with
    DataFormat VTK and DataWriteFreq 200, steps 0, 200, 400, 401."""
    import hashlib
    from _oracle import Oracle
    from conftest import golden
    want = golden("vtk_small4")["files"]
    p = M.read_deck(golden_deck("small4"))
    o = Oracle(p)
    import os
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        for ts in (0, 200, 400, 401):
            o.step(ts - o.timestep)
            M.write_vtk_arrays(p, "small4", ts, o.download("temperature"), o.download("gr"))
    finally:
        os.chdir(cwd)
    got = {str(f.relative_to(tmp_path)): hashlib.sha256(f.read_bytes()).hexdigest()
           for f in sorted(tmp_path.rglob("*")) if f.suffix in (".vtu", ".pvtu")}
    assert got == want


@pytest.mark.gpu
def test_vtk_from_device(built, cuda_device, tmp_path):
    p = M.read_deck(golden_deck("small1"))
    with M.Domain(p) as dom:
        dom.step(100)
        base = str(tmp_path / "dev")
        dom.write_vtk(base)
        piece = next(ET.parse(f"{base}_0000/100.vtu").getroot().iter("Piece"))
        grain = _decode(_arr(piece, "Grain"))
        gr = dom.download("gr")[1:-1, 1:-1, 1:-1]
        assert np.array_equal(grain, np.transpose(gr, (2, 1, 0)).ravel())


# ---------------------------------------------------------------- XDMF
def _xdmf_item(d: Path, item) -> np.ndarray:
    """A Format="Binary" DataItem of the index, read from its raw file."""
    dt = {("Float", "4"): "<f4", ("Int", "4"): "<i4", ("UInt", "8"): "<u8"}[(item.get("NumberType"),
                                                                          item.get("Precision"))]
    dims = tuple(int(x) for x in item.get("Dimensions").split())
    n = int(np.prod(dims))
    return np.fromfile(d / item.text.strip(), dtype=dt, count=n, offset=int(item.get("Seek"))).reshape(dims)


def _check_xdmf(tmp: Path, base: str, p, series, fields, rotang, renumber):
    """Index structure (io_xdmf.c:141-305, 378-404) and every dataset against
    the halo'd arrays it was written from (fields: name -> [z, y, x])."""
    import xml.etree.ElementTree as ET
    root = ET.parse(tmp / f"{base}_ts.xmf").getroot()
    dom = root.find("Domain")
    series_grid = dom.find("Grid")
    assert series_grid.get("CollectionType") == "Temporal"
    grids = series_grid.findall("Grid")
    assert len(grids) == len(series)
    nsub = p.gnsbx * p.gnsby * p.gnsbz
    sd = (p.gsdimz, p.gsdimy, p.gsdimx)
    glob = {it.get("Name"): it for it in dom.findall("DataItem")}
    for d, ax in enumerate("XYZ"):
        np.testing.assert_array_equal(_xdmf_item(tmp, glob[f"Grain Angle {ax}"]),
                                      rotang[:, d].astype(np.float32))
    if renumber is not None:
        np.testing.assert_array_equal(_xdmf_item(tmp, glob["Grain Renumber"]), renumber)
    else:
        assert "Grain Renumber" not in glob
    last = grids[-1]
    assert float(last.find("Time").get("Value")) == pytest.approx(series[-1] * p.ts_delt)
    blocks = last.findall("Grid")
    assert len(blocks) == nsub
    for s, g in enumerate(blocks):
        cx, cy, cz = s % p.gnsbx, (s // p.gnsbx) % p.gnsby, s // (p.gnsbx * p.gnsby)
        assert g.get("Name") == f"SubBlock {cx}x{cy}x{cz} ({s})"
        assert g.find("Topology").get("Dimensions") == f"{sd[0] + 1} {sd[1] + 1} {sd[2] + 1}"
        origin = [float(v) for v in g.find("Geometry").findall("DataItem")[0].text.split()]
        want = [p.origin_offset[2] + cz * sd[0] * p.cellSize, p.origin_offset[1] + cy * sd[1] * p.cellSize,
                p.origin_offset[0] + cx * sd[2] * p.cellSize]
        assert origin == pytest.approx(want, rel=1e-5, abs=1e-12)
        sl = (slice(cz * sd[0] + 1, (cz + 1) * sd[0] + 1), slice(cy * sd[1] + 1, (cy + 1) * sd[1] + 1),
              slice(cx * sd[2] + 1, (cx + 1) * sd[2] + 1))
        att = {a.get("Name"): a for a in g.findall("Attribute")}
        for name, key, dt in (("Temperature", "temperature", np.float32), ("Solute Composition", "ce", np.float32),
                              ("Fraction Solid", "fs", np.float32)):
            np.testing.assert_array_equal(_xdmf_item(tmp, att[name].find("DataItem")), fields[key][sl].astype(dt))
        grain_item = att["Grain"].find(".//DataItem[@Format='Binary']")
        np.testing.assert_array_equal(_xdmf_item(tmp, grain_item), fields["gr"][sl])
        fn = att["Grain"].find("DataItem")
        assert (fn.get("ItemType") == "Function") == (renumber is not None)


def test_xdmf_arrays_layout(built, tmp_path):
    """Two writes of a 2 x 1 x 2 subblock deck from host arrays: the index
    lists both timesteps; every dataset of the second one reads back."""
    p = M.default_params()
    p.gnsbx, p.gnsby, p.gnsbz = 2, 1, 2
    p.gsdimx, p.gsdimy, p.gsdimz = 5, 4, 3
    p.cellSize, p.ts_delt = 2e-6, 1e-4
    nx, ny, nz = (v + 2 for v in p.grid)
    rng = np.random.default_rng(3)
    f = {"temperature": rng.normal(900, 5, (nz, ny, nx)), "ce": rng.random((nz, ny, nx)),
         "fs": rng.random((nz, ny, nx)), "gr": rng.integers(0, 7, (nz, ny, nx)).astype(np.int32)}
    rot = rng.normal(size=(7, 3))
    ren = rng.permutation(7).astype(np.uint64)
    base = str(tmp_path / "xd")
    for series in ([0], [0, 10]):
        M.write_xdmf_arrays(p, base, series, f["temperature"], f["ce"], f["gr"], f["fs"], rot, ren)
    _check_xdmf(tmp_path, "xd", p, [0, 10], f, rot, ren)
    M.write_xdmf_arrays(p, base, [0], f["temperature"], f["ce"], f["gr"], f["fs"], rot, None)
    _check_xdmf(tmp_path, "xd", p, [0], f, rot, None)


def test_oracle_xdmf_renumbering_shifts_rank0_draws(built):
    """The reference's XDMF writer draws its grain renumbering from rank 0's
    rand() stream (io_xdmf.c:344-375): a permutation fixing 0, redrawn only
    when the grain count grew, and later orientation draws of rank 0 follow
    it, so the same deck with XDMF writes evolves differently."""
    from _oracle import Oracle
    p = M.read_deck(golden_deck("small4"))
    a, b = Oracle(p), Oracle(p)
    for s in (60, 120, 180, 260):
        a.step(s - a.timestep)
        b.step(s - b.timestep)
        if s < 260:
            r = a.xdmf_renumber()
            assert r[0] == 0 and sorted(r.tolist()) == list(range(a.num_grains))
            assert np.array_equal(a.xdmf_renumber(), r)  # same grain count: no new draws
    assert mismatches(state_digests(a), state_digests(b))


@pytest.mark.gpu
def test_xdmf_writes_bit_exact_vs_oracle(built, cuda_device, tmp_path):
    """small4 with XDMF writes at steps 60, 120, 180 (RandomizeGrains 1):
    the device run's renumberings equal the oracle's, its state stays
    bit-identical to the oracle's through step 260, and the files of the last
    write hold the device fields."""
    from _oracle import Oracle
    p = M.read_deck(golden_deck("small4"))
    o = Oracle(p)
    base = str(tmp_path / "s4")
    with M.Domain(p, precision=M.PREC_F64) as dom:
        for s in (60, 120, 180, 260):
            o.step(s - o.timestep)
            dom.step(s - dom.timestep)
            assert mismatches(state_digests(dom), state_digests(o)) == [], s
            if s < 260:
                dom.write_xdmf(base)
                np.testing.assert_array_equal(dom.xdmf_renumbering(), o.xdmf_renumber())
                if s == 180:
                    fields = {k: dom.download(k) for k in ("temperature", "ce", "fs", "gr")}
                    rot = np.array([list(g.rotang) for g in dom.grains()])
                    _check_xdmf(tmp_path, "s4", p, [60, 120, 180], fields, rot, dom.xdmf_renumbering())
        assert dom.num_grains == o.num_grains


@pytest.mark.gpu
def test_run_loop_writes_xdmf_like_reference(built, cuda_device, tmp_path):
    """mms_run on small4 with DataFormat XDMF and DataWriteFreq 100: writes
    at steps 0, 100, ..., 400 and at the last step, 401 (FinishTime 0.4005;
    writeData, loop.c:199-256), the index lists them all, and the end state
    equals the oracle stepped with the same renumberings."""
    from _oracle import Oracle
    text = golden_deck("small4").read_text()
    text = "\n".join(l for l in text.splitlines() if not l.startswith("BaseFileName"))
    text += f"\nBaseFileName {tmp_path}/r4\nDataFormat XDMF\nDataWriteFreq 100\n"
    deck = tmp_path / "r4.in"
    deck.write_text(text)
    p = M.read_deck(deck)
    o = Oracle(p)
    o.xdmf_renumber()
    for s in (100, 200, 300, 400, 401):
        o.step(s - o.timestep)
        o.xdmf_renumber()
    with M.Domain(p, precision=M.PREC_F64) as dom:
        dom.run(verbose=0)
        assert dom.timestep == 401
        assert mismatches(state_digests(dom), state_digests(o)) == []
        np.testing.assert_array_equal(dom.xdmf_renumbering(), o.xdmf_renumber())
    import xml.etree.ElementTree as ET
    grids = ET.parse(tmp_path / "r4_ts.xmf").getroot().find("Domain").find("Grid").findall("Grid")
    times = [round(float(g.find("Time").get("Value")) / p.ts_delt) for g in grids]
    assert times == [0, 100, 200, 300, 400, 401]
    assert (tmp_path / "r4_r3" / "00401.raw").exists()


@pytest.mark.gpu
def test_run_loop_writes_vtk(built, cuda_device, tmp_path):
    """mms_run with DataFormat VTK and DataWriteFreq 200 on small4 (to step
    401): ParaView files at steps 0, 200, 400 and 401 (writeData,
    loop.c:199-256), one piece per subblock, the last holding the end state."""
    text = golden_deck("small4").read_text()
    text = "\n".join(l for l in text.splitlines() if not l.startswith("BaseFileName"))
    text += f"\nBaseFileName {tmp_path}/v4\nDataFormat VTK\nDataWriteFreq 200\n"
    deck = tmp_path / "v4.in"
    deck.write_text(text)
    p = M.read_deck(deck)
    with M.Domain(p, precision=M.PREC_F64) as dom:
        dom.run(verbose=0)
        gr = dom.download("gr")
    for ts in (0, 200, 400, 401):
        assert (tmp_path / f"v4_{ts}.pvtu").exists(), ts
    nsub = p.gnsbx * p.gnsby * p.gnsbz
    piece = ET.parse(tmp_path / "v4_0000" / "401.vtu").getroot()
    got = _decode(_arr(piece, "Grain"))
    sd = (p.gsdimz, p.gsdimy, p.gsdimx)
    # subblock 0, cells in the reference's x-major order (x outer, z inner)
    want = gr[1:sd[0] + 1, 1:sd[1] + 1, 1:sd[2] + 1].transpose(2, 1, 0).reshape(-1)
    assert nsub == 4 and np.array_equal(got, want)


@pytest.mark.gpu
def test_run_loop_vtk_bytes_match_reference(built, cuda_device, tmp_path):
    """mmsb200's run loop on small4 with DataFormat VTK writes the very files
    the reference writes (digests recorded from the reference itself)."""
    import hashlib
    import os
    from conftest import golden
    want = golden("vtk_small4")["files"]
    deck = _vtk_deck(tmp_path)
    p = M.read_deck(deck)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        with M.Domain(p, precision=M.PREC_F64) as dom:
            dom.run(verbose=0)
    finally:
        os.chdir(cwd)
    got = {str(f.relative_to(tmp_path)): hashlib.sha256(f.read_bytes()).hexdigest()
           for f in sorted(tmp_path.rglob("*")) if f.suffix in (".vtu", ".pvtu")}
    assert got == want
