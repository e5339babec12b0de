"""ctypes binding of the CPU oracle (oracle/mms_oracle.c) — test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
this; the product never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
LIB_PATH = ORACLE_DIR / "_ref" / "liboracle.so"
REF_BIN = ORACLE_DIR / "_ref" / "mmsref"

_LIB = None


def load():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        subprocess.run(["make", "-C", str(ORACLE_DIR), "oracle"], check=True, capture_output=True)
    from mumatscale_b200 import Params, Grain, GrainSummary
    lib = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    lib.mmso_create.restype = P
    lib.mmso_create.argtypes = [C.POINTER(Params), C.POINTER(C.c_int)]
    lib.mmso_destroy.argtypes = [P]
    lib.mmso_set_sites.argtypes = [P, C.c_int64, P, P]
    lib.mmso_set_site_orientations.argtypes = [P, C.c_int64, P, P]
    lib.mmso_set_grains.argtypes = [P, C.c_int, P]
    lib.mmso_set_field.argtypes = [P, C.c_int, P]
    lib.mmso_enable_curvature.argtypes = [P, C.c_int]
    lib.mmso_step.argtypes = [P, C.c_int]
    lib.mmso_timestep.restype = C.c_uint64
    lib.mmso_timestep.argtypes = [P]
    lib.mmso_num_grains.argtypes = [P]
    lib.mmso_num_cells.restype = C.c_size_t
    lib.mmso_num_cells.argtypes = [P]
    lib.mmso_get_field.argtypes = [P, C.c_int, P]
    lib.mmso_reduce.restype = C.c_double
    lib.mmso_reduce.argtypes = [P, C.c_int]
    lib.mmso_get_grains.argtypes = [P, C.c_int, C.c_int, C.POINTER(Grain)]
    lib.mmso_grain_summary.argtypes = [P, C.POINTER(GrainSummary)]
    lib.mmso_run.argtypes = [P, C.c_int]
    lib.mmso_rand_sequence.argtypes = [C.c_uint, C.c_int, P]
    lib.mmso_xdmf_renumber.argtypes = [P, P, C.c_int]
    _LIB = lib
    return lib


_DT = {0: (np.float64, 1), 1: (np.float64, 1), 2: (np.float64, 1), 3: (np.int32, 1),
       4: (np.float64, 3), 5: (np.float64, 1), 6: (np.float32, 1), 7: (np.float64, 1),
       8: (np.int8, 1), 9: (np.int32, 1), 10: (np.float64, 1)}
FIELD = {"ce": 0, "cl": 1, "fs": 2, "gr": 3, "dc": 4, "d": 5, "nuc_threshold": 6,
         "temperature": 7, "mold": 8, "ogr": 9, "curv": 10}


class Oracle:
    def __init__(self, params, curvature: bool = False):
        lib = load()
        st = C.c_int()
        self._o = lib.mmso_create(C.byref(params), C.byref(st))
        if not self._o:
            raise RuntimeError(f"mmso_create failed with status {st.value}")
        self.shape = tuple(x + 2 for x in params.grid)
        if curvature:
            lib.mmso_enable_curvature(self._o, 1)

    def close(self):
        if self._o:
            load().mmso_destroy(self._o)
            self._o = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        st = load().mmso_step(self._o, int(n))
        if st:
            raise RuntimeError(f"oracle step failed with status {st}")

    def run(self, verbose=0):
        return load().mmso_run(self._o, int(verbose))

    def set_sites(self, gxyz, thr):
        g = np.ascontiguousarray(gxyz, dtype=np.int32).reshape(-1, 3)
        t = np.ascontiguousarray(thr, dtype=np.float32).reshape(-1)
        st = load().mmso_set_sites(self._o, len(t), g.ctypes.data, t.ctypes.data)
        if st:
            raise RuntimeError(f"oracle set_sites failed with status {st}")

    def set_site_orientations(self, gxyz, rot):
        g = np.ascontiguousarray(gxyz, dtype=np.int32).reshape(-1, 3)
        r = np.ascontiguousarray(rot, dtype=np.float64).reshape(-1, 9)
        load().mmso_set_site_orientations(self._o, len(r), g.ctypes.data, r.ctypes.data)

    def set_grains(self, rot):
        r = np.ascontiguousarray(rot, dtype=np.float64).reshape(-1, 9)
        st = load().mmso_set_grains(self._o, len(r), r.ctypes.data)
        if st:
            raise RuntimeError(f"mmso_set_grains failed with status {st}")

    def upload(self, name, arr):
        from mumatscale_b200 import FIELD
        dt = np.int32 if name == "gr" else np.float64
        a = np.ascontiguousarray(arr, dtype=dt)
        st = load().mmso_set_field(self._o, FIELD[name], a.ctypes.data)
        if st:
            raise RuntimeError(f"mmso_set_field failed with status {st}")

    @property
    def timestep(self):
        return int(load().mmso_timestep(self._o))

    @property
    def num_grains(self):
        return int(load().mmso_num_grains(self._o))

    def download(self, name):
        f = FIELD[name]
        dt, comp = _DT[f]
        n = int(load().mmso_num_cells(self._o))
        out = np.empty(n * comp, dtype=dt)
        load().mmso_get_field(self._o, f, out.ctypes.data)
        nx, ny, nz = self.shape
        return out.reshape((nz, ny, nx, comp) if comp > 1 else (nz, ny, nx))

    def xdmf_renumber(self) -> np.ndarray:
        """The reference XDMF writer's grain renumbering (rank 0's stream)."""
        n = load().mmso_xdmf_renumber(self._o, None, 0)
        out = np.empty(n, dtype=np.uint64)
        load().mmso_xdmf_renumber(self._o, out.ctypes.data, n)
        return out

    def reduce(self, what="fs_fraction"):
        return float(load().mmso_reduce(self._o, {"fs_fraction": 0, "solid_volume": 1, "ce_sum": 2}[what]))

    def grains(self):
        from mumatscale_b200 import Grain
        n = self.num_grains
        arr = (Grain * n)()
        load().mmso_get_grains(self._o, 0, n, arr)
        return list(arr)

    def grain_summary(self):
        from mumatscale_b200 import GrainSummary
        s = GrainSummary()
        load().mmso_grain_summary(self._o, C.byref(s))
        return s


def rand_sequence(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.int32)
    load().mmso_rand_sequence(seed, n, out.ctypes.data)
    return out
