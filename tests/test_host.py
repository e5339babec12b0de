"""Host-side logic that needs no GPU: the C-ABI library loads and exports
every entry point include/mms.h declares, the mms_params layout agrees with
the binding, and the deck parser follows read_ctrl.c."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

import mumatscale_b200 as M
from conftest import ROOT, golden_deck

HEADER = ROOT / "include" / "mms.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mms_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(built):
    lib = M.load_library()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(M.library_path())], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (mms_\w+)", out))
    assert set(names) <= exported


def test_params_layout(built):
    lib = M.load_library()
    assert lib.mms_params_size() == C.sizeof(M.Params)


def test_defaults_follow_set_defaults(built):
    p = M.default_params()
    assert p.cellSize == float(C.c_float(0.01).value)  # 0.01f literal, read_ctrl.c:37
    assert p.ts_delt == float(C.c_float(0.1).value)
    assert p.liquidusTemp == 1180.0 and p.courant_limit == 0.2
    assert p.maxTotalGrains == 1000000 and p.doSurfaceNuc == 1 and p.screenpfreq == 1
    assert p.part_coef == 0.3 and p.m_solute0 == -2.0 and p.Cinit == 5.0
    assert (p.padBndyX, p.padBndyY, p.padBndyZ) == (1, 1, 1)
    assert p.basefilename == b"output"


def test_deck_one_grain(built):
    p = M.read_deck(golden_deck("small1"))
    assert (p.gnsbx, p.gnsby, p.gnsbz) == (1, 1, 1)
    assert (p.gsdimx, p.gsdimy, p.gsdimz) == (20, 18, 16)
    assert p.cellSize == 5e-6 and p.ts_delt == 1e-3 and p.base_random_seed == 12345
    assert p.fsgrow == 0.66 and p.rev_fsgrow == 1.0 / 0.66
    assert p.m_solute0 == -10.9 and p.part_coef == 0.67
    assert p.n_fixed_nucs == 1
    f = p.fixed_nucs[0]
    assert (f.x, f.y, f.z, f.ax, f.ay, f.az, f.threshold) == (5.25e-5, 4.75e-5, 4.25e-5, 10, 20, 30, 0.5)
    assert p.gnUseOrientation == 1 and p.maxTotalGrains == 100000


def test_deck_quirks(built, tmp_path: Path):
    inc = tmp_path / "mat.in"
    inc.write_text("Dliq 4e-9  /* trailing comment ignored by sscanf */\nCinit 3.3\n")
    deck = tmp_path / "main.in"
    deck.write_text(
        "# comment\n% also comment\n"
        "nsubblocks 2 1 3\nNCELLSPERSB 4 5 6\n"
        f"MatFileName {inc}\n"
        "DataWriteStart 7\n"
        "UnknownKeyword 12\n"
        "NucVolume 50 0 0 0 1e-5 1e-5 1e-5 0.3\n"
        "AnalyticalThermal 1\n")
    p = M.read_deck(deck)
    assert (p.gnsbx, p.gnsby, p.gnsbz, p.gsdimx, p.gsdimy, p.gsdimz) == (2, 1, 3, 4, 5, 6)
    assert p.Dliq == 4e-9 and p.Cinit == 3.3
    assert p.data_write_start == 7
    assert p.n_nuc_volumes == 1 and p.nuc_volumes[0].density == 0.5
    assert p.am == 1 and p.thermal_ana == 1


@pytest.mark.parametrize("line", ["CalculationModel DIFFUSION", "TemperatureModel EXTERNAL",
                                  "DataFormat NONE", "NSubblocks 1 2", "FaceCtrl 1 0 1 1 1 1"])
def test_deck_errors(built, tmp_path: Path, line):
    deck = tmp_path / "bad.in"
    deck.write_text(line + "\n")
    with pytest.raises(M.MmsError) as e:
        M.read_deck(deck)
    assert e.value.status == 7  # MMS_ERR_DECK


def test_missing_deck(built, tmp_path: Path):
    with pytest.raises(M.MmsError):
        M.read_deck(tmp_path / "nope.in")


def test_create_without_device_fails_loudly(built):
    """No silent CPU fallback: without a CUDA device mms_create refuses."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except Exception:
        pass
    p = M.read_deck(golden_deck("small1"))
    with pytest.raises(M.MmsError) as e:
        M.Domain(p)
    assert e.value.status == 3  # MMS_ERR_NO_DEVICE


def test_courant_check(built):
    p = M.read_deck(golden_deck("small1"))
    p.ts_delt = 1.0  # Dliq dt / dx^2 = 120 > 0.2
    with pytest.raises(M.MmsError) as e:
        M.Domain(p)
    assert e.value.status in (3, 4)  # no device here, or MMS_ERR_COURANT


@pytest.mark.parametrize("name", ["small1", "small4", "nucvol1", "grad1", "am1", "cap1"])
def test_predraw_sites_matches_reference(built, name):
    """The product's host-side replay of the reference's site draws
    (mms_predraw_sites) reproduces the reference's threshold field."""
    from conftest import golden
    from digests import digest
    rec = golden(name)
    p = M.read_deck(golden_deck(name))
    assert digest(M.predraw_sites(p)) == rec["setup"]["nuc_threshold"]
