"""mumatscale_b200 — B200-native muMatScale CA solidification step.

The compute lives in the in-tree C-ABI library ``libmms_b200.so``
(include/mms.h): hand-written sm_100a kernels plus their host side.  This
module only binds that library with ctypes and mirrors the reference's
interfaces: an input deck (read_ctrl.c) becomes :class:`Params`, a
:class:`Domain` owns the device-resident fields of one GPU and advances
them by whole timesteps (doiteration, calculate.c:193-352), and
:meth:`Domain.run` is the reference time loop (loop.c:186-271).

There is no CPU fallback: if the library or a CUDA device is missing, the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

__all__ = [
    "Params", "FixedNuc", "NucVolume", "Grain", "GrainSummary", "Domain", "MmsError",
    "load_library", "library_path", "FIELD", "PREC_F64", "PREC_F32",
    "Batch", "SlabLayout", "SlabDomain", "SlabGroup", "slab_layout",
]

_PKG = Path(__file__).resolve().parent
PREC_F64 = 0
PREC_F32 = 1

FIELD = {
    "ce": 0, "cl": 1, "fs": 2, "gr": 3, "dc": 4, "d": 5,
    "nuc_threshold": 6, "temperature": 7, "mold": 8, "ogr": 9, "curv": 10,
}
_FIELD_DTYPE = {
    0: (np.float64, 1), 1: (np.float64, 1), 2: (np.float64, 1), 3: (np.int32, 1),
    4: (np.float64, 3), 5: (np.float64, 1), 6: (np.float32, 1), 7: (np.float64, 1),
    8: (np.int8, 1), 9: (np.int32, 1), 10: (np.float64, 1),
}
REDUCE = {"fs_fraction": 0, "solid_volume": 1, "ce_sum": 2}


class FixedNuc(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("x", "y", "z", "ax", "ay", "az", "threshold")]


class NucVolume(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("density", "minx", "miny", "minz", "maxx", "maxy", "maxz", "threshold")]


class AdjointResult(C.Structure):
    _fields_ = [("loss", C.c_double), ("dL_dDliq", C.c_double), ("dL_dpart_coef", C.c_double),
                ("dL_dgibbs", C.c_double), ("steps", C.c_int64)]


class Params(C.Structure):
    """mms_params: the BB_struct subset (globals.h:273-403) the hot path reads."""
    _fields_ = [
        ("gnsbx", C.c_int), ("gnsby", C.c_int), ("gnsbz", C.c_int),
        ("gsdimx", C.c_int), ("gsdimy", C.c_int), ("gsdimz", C.c_int),
        ("padBndyX", C.c_int), ("padBndyY", C.c_int), ("padBndyZ", C.c_int),
        ("origin_offset", C.c_double * 3),
        ("cellSize", C.c_double), ("courant_limit", C.c_double),
        ("base_random_seed", C.c_uint),
        ("ts_delt", C.c_double), ("finish_time", C.c_double), ("fs_finish", C.c_double),
        ("fsgrow", C.c_double), ("rev_fsgrow", C.c_double),
        ("tip_curv", C.c_int), ("gibbs_coef", C.c_double),
        ("liquidusTemp", C.c_double), ("solidusTemp", C.c_double), ("Cinit", C.c_double),
        ("m_solute0", C.c_double), ("m_solute0_a", C.c_double), ("m_solute0_b", C.c_double),
        ("m_solute0_c", C.c_double),
        ("part_coef", C.c_double), ("part_coef_a", C.c_double), ("part_coef_b", C.c_double),
        ("part_coef_c", C.c_double),
        ("Dsol", C.c_double), ("Dliq", C.c_double),
        ("initialTemperature", C.c_double), ("gradient", C.c_double), ("velocity", C.c_double),
        ("grad_coef", C.c_double), ("velo_coef", C.c_double), ("cool_rate", C.c_double),
        ("thermal_ana", C.c_int), ("am", C.c_int), ("amlayer", C.c_int), ("amtracks", C.c_int),
        ("lpow", C.c_double), ("lv", C.c_double), ("lsd", C.c_double), ("lab", C.c_double),
        ("lhs", C.c_double), ("liniT", C.c_double), ("lthcon", C.c_double), ("lcp", C.c_double),
        ("rho", C.c_double), ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double),
        ("maxGrainDensity", C.c_double), ("gnGaussCenter", C.c_double),
        ("gnGaussSigma", C.c_double),
        ("maxGrainDensitySurf", C.c_double), ("gnGaussCenterSurf", C.c_double),
        ("gnGaussSigmaSurf", C.c_double),
        ("doSurfaceNuc", C.c_int), ("gnUseOrientation", C.c_int),
        ("maxTotalGrains", C.c_uint64),
        ("screenpfreq", C.c_int), ("data_write_freq", C.c_int), ("data_write_start", C.c_int),
        ("randomize_grains", C.c_int), ("vis_format", C.c_int),
        ("basefilename", C.c_char * 256),
        ("fixed_nucs", C.POINTER(FixedNuc)), ("n_fixed_nucs", C.c_int),
        ("nuc_volumes", C.POINTER(NucVolume)), ("n_nuc_volumes", C.c_int),
        ("precision", C.c_int), ("device", C.c_int), ("site_setup", C.c_int),
        ("checkpoint_freq", C.c_int), ("curvature_corrected", C.c_int),
    ]

    @property
    def grid(self) -> tuple[int, int, int]:
        return (self.gnsbx * self.gsdimx, self.gnsby * self.gsdimy, self.gnsbz * self.gsdimz)

    @property
    def nranks(self) -> int:
        return self.gnsbx * self.gnsby * self.gnsbz


class Grain(C.Structure):
    """grain_t (globals.h:244-254)."""
    _fields_ = [("nuc_x", C.c_double), ("nuc_y", C.c_double), ("nuc_z", C.c_double),
                ("nuc_timestep", C.c_uint64), ("nuc_threshold", C.c_double),
                ("rotmat", (C.c_double * 3) * 3), ("rotang", C.c_double * 3)]


class SlabLayout(C.Structure):
    """mms_slab_layout: the z-range and emulated ranks one slab owns."""
    _fields_ = [("nslabs", C.c_int), ("slab", C.c_int), ("z_begin", C.c_int), ("z_cells", C.c_int),
                ("rank_begin", C.c_int), ("rank_count", C.c_int)]


class SlabXfer(C.Structure):
    """mms_slab_xfer: one transfer of a slab exchange point."""
    _fields_ = [("kind", C.c_int), ("peer", C.c_int), ("send", C.c_void_p), ("recv", C.c_void_p),
                ("bytes", C.c_uint64)]


XFER_HALO = 0
XFER_GATHER = 1


class GrainSummary(C.Structure):
    _fields_ = [("num_grains", C.c_int), ("min_mm3", C.c_double), ("max_mm3", C.c_double),
                ("avg_mm3", C.c_double)]


class MmsError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where}: {_lib().mms_status_string(status).decode()} (status {status})"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


_LIB = None


def library_path() -> Path:
    """The in-tree libmms_b200.so, or the library MMS_LIBRARY names (for
    instance the bounds-checked build, libmms_b200_bounds.so)."""
    alt = os.environ.get("MMS_LIBRARY")
    return Path(alt) if alt else _PKG / "libmms_b200.so"


def load_library(build_if_missing: bool = True) -> C.CDLL:
    """Loads libmms_b200.so from the package directory (building it first
    when it is missing and nvcc is available)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not path.exists() and build_if_missing:
        from . import build as _build
        _build.build()
    if not path.exists():
        raise OSError(f"{path} is missing; run `python -m mumatscale_b200.build`")
    lib = C.CDLL(str(path))
    P, I, D = C.c_void_p, C.c_int, C.c_double
    sigs = {
        "mms_params_default": (I, [C.POINTER(Params)]),
        "mms_deck_read": (I, [C.c_char_p, C.POINTER(Params)]),
        "mms_params_free_lists": (None, [C.POINTER(Params)]),
        "mms_params_size": (C.c_size_t, []),
        "mms_test_hold_list_block": (I, [P, I, C.c_uint]),
        "mms_slab_nccl_unique_id": (I, [C.c_char_p, P]),
        "mms_slab_nccl_init": (I, [P, C.c_char_p, P]),
        "mms_slab_nccl_step": (I, [P, I]),
        "mms_slab_nccl_reduce": (I, [P, I, C.POINTER(D)]),
        "mms_create": (I, [C.POINTER(Params), C.POINTER(P)]),
        "mms_destroy": (I, [P]),
        "mms_step": (I, [P, I]),
        "mms_get_timestep": (I, [P, C.POINTER(C.c_uint64)]),
        "mms_get_num_grains": (I, [P, C.POINTER(I)]),
        "mms_num_cells": (C.c_size_t, [P]),
        "mms_download": (I, [P, I, P]),
        "mms_upload": (I, [P, I, P]),
        "mms_reduce": (I, [P, I, C.POINTER(D)]),
        "mms_step_reduce": (I, [P, I, I, C.POINTER(D)]),
        "mms_set_sites": (I, [P, C.c_int64, P, P]),
        "mms_set_site_orientations": (I, [P, C.c_int64, P, P]),
        "mms_get_grains": (I, [P, I, I, C.POINTER(Grain)]),
        "mms_output_grains": (I, [P, C.c_char_p, C.POINTER(GrainSummary)]),
        "mms_run": (I, [P, I]),
        "mms_status_string": (C.c_char_p, [I]),
        "mms_last_error": (C.c_char_p, [P]),
        "mms_kernel_launches": (C.c_uint64, [P]),
        "mms_uses_tma": (I, [P]),
        "mms_predraw_sites": (I, [C.POINTER(Params), P]),
        "mms_set_stream": (I, [P, P]),
        "mms_set_profiling": (I, [P, I]),
        "mms_kernel_count": (I, []),
        "mms_kernel_name": (C.c_char_p, [I]),
        "mms_kernel_stats": (I, [P, I, C.POINTER(D), C.POINTER(C.c_uint64)]),
        "mms_set_stencil_tile": (I, [P, I, I]),
        "mms_get_stencil_tile": (I, [P, C.POINTER(I), C.POINTER(I)]),
        "mms_set_am_tile": (I, [P, I]),
        "mms_get_am_tile": (I, [P, C.POINTER(I)]),
        "mms_autotune": (I, [P, I, C.POINTER(I), C.POINTER(I), C.POINTER(D)]),
        "mms_adjoint_record": (I, [P, I, I]),
        "mms_adjoint_gradient": (I, [P, P, C.POINTER(AdjointResult)]),
        "mms_adjoint_replay_loss": (I, [P, P, C.POINTER(D), C.POINTER(D)]),
        "mms_adjoint_release": (I, [P]),
        "mms_set_grains": (I, [P, I, P]),
        "mms_write_vtk": (I, [P, C.c_char_p]),
        "mms_checkpoint_save": (I, [P, C.c_char_p]),
        "mms_checkpoint_load": (I, [P, C.c_char_p]),
        "mms_write_vtk_arrays": (I, [C.POINTER(Params), C.c_char_p, C.c_int64, P, P]),
        "mms_batch_create": (I, [I, C.POINTER(Params), C.POINTER(P)]),
        "mms_batch_destroy": (I, [P]),
        "mms_batch_size": (I, [P]),
        "mms_batch_domain": (P, [P, I]),
        "mms_batch_step": (I, [P, I]),
        "mms_batch_set_stencil_tile": (I, [P, I, I]),
        "mms_batch_get_stencil_tile": (I, [P, C.POINTER(I), C.POINTER(I), C.POINTER(I)]),
        "mms_batch_autotune": (I, [P, I, C.POINTER(I), C.POINTER(I), C.POINTER(D)]),
        "mms_batch_kernel_launches": (C.c_uint64, [P]),
        "mms_batch_last_error": (C.c_char_p, [P]),
        "mms_write_xdmf": (I, [P, C.c_char_p]),
        "mms_write_xdmf_arrays": (I, [C.POINTER(Params), C.c_char_p, P, I, P, P, P, P, I, P, P]),
        "mms_xdmf_renumbering": (I, [P, I, P, C.POINTER(I)]),
        "mms_slab_layout_of": (I, [C.POINTER(Params), I, I, C.POINTER(SlabLayout)]),
        "mms_slab_create": (I, [C.POINTER(Params), I, I, C.POINTER(P)]),
        "mms_slab_get_layout": (I, [P, C.POINTER(SlabLayout)]),
        "mms_slab_group_step": (I, [C.POINTER(P), I, I]),
        "mms_slab_launch": (I, [P, I, I]),
        "mms_slab_exchange_plan": (I, [P, I, C.c_uint64, C.POINTER(SlabXfer), I, C.POINTER(I)]),
        "mms_slab_poll": (I, [P, C.POINTER(C.c_uint64), C.POINTER(I)]),
        "mms_slab_refill": (I, [P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.mms_params_size() != C.sizeof(Params):
        raise OSError(f"mms_params layout mismatch: C {lib.mms_params_size()} vs "
                      f"ctypes {C.sizeof(Params)}")
    _LIB = lib
    return lib


def _lib() -> C.CDLL:
    return load_library()


def _check(status: int, where: str, ctx=None) -> None:
    if status != 0:
        detail = ""
        if ctx:
            detail = (_lib().mms_last_error(ctx) or b"").decode()
        raise MmsError(status, where, detail)


def write_vtk_arrays(params: Params, base: str, timestep: int, temperature: np.ndarray, gr: np.ndarray) -> None:
    """ParaView files (io_vtk.c layout) from halo'd host arrays."""
    t = np.ascontiguousarray(temperature, dtype=np.float64)
    g = np.ascontiguousarray(gr, dtype=np.int32)
    _check(_lib().mms_write_vtk_arrays(C.byref(params), base.encode(), timestep, t.ctypes.data, g.ctypes.data),
           "mms_write_vtk_arrays")


def write_xdmf_arrays(params: Params, base: str, series, temperature: np.ndarray, ce: np.ndarray,
                      gr: np.ndarray, fs: np.ndarray, rotang: np.ndarray, renumber: np.ndarray | None = None) -> None:
    """XDMF files (io_xdmf.c layout, raw binary datasets) from halo'd host
    arrays; series: the time series' timesteps, the last being this write's."""
    ser = np.ascontiguousarray(series, dtype=np.int64)
    t = np.ascontiguousarray(temperature, dtype=np.float64)
    c = np.ascontiguousarray(ce, dtype=np.float64)
    g = np.ascontiguousarray(gr, dtype=np.int32)
    f = np.ascontiguousarray(fs, dtype=np.float64)
    a = np.ascontiguousarray(rotang, dtype=np.float64).reshape(-1, 3)
    r = None if renumber is None else np.ascontiguousarray(renumber, dtype=np.uint64)
    _check(_lib().mms_write_xdmf_arrays(C.byref(params), base.encode(), ser.ctypes.data, len(ser), t.ctypes.data,
                                        c.ctypes.data, g.ctypes.data, f.ctypes.data, len(a), a.ctypes.data,
                                        None if r is None else r.ctypes.data), "mms_write_xdmf_arrays")


def default_params() -> Params:
    """set_defaults (read_ctrl.c:29-108)."""
    p = Params()
    _check(_lib().mms_params_default(C.byref(p)), "mms_params_default")
    return p


def read_deck(path: str | os.PathLike, params: Params | None = None) -> Params:
    """read_config (read_ctrl.c:234-812) on top of defaults (or ``params``)."""
    p = params if params is not None else default_params()
    _check(_lib().mms_deck_read(str(path).encode(), C.byref(p)), f"mms_deck_read({path})")
    return p


def predraw_sites(params: Params) -> np.ndarray:
    """The reference's threshold field after setup, computed on the host
    (no device needed); shape (z, y, x) of the halo'd grid."""
    nx, ny, nz = (x + 2 for x in params.grid)
    out = np.empty(nx * ny * nz, dtype=np.float32)
    _check(_lib().mms_predraw_sites(C.byref(params), out.ctypes.data), "mms_predraw_sites")
    return out.reshape(nz, ny, nx)


Params.default = staticmethod(default_params)
Params.from_deck = staticmethod(read_deck)


class Domain:
    """One GPU's device-resident domain (one mms_ctx)."""

    def __init__(self, params: Params, precision: int | None = None, device: int | None = None):
        lib = _lib()
        p = Params()
        C.pointer(p)[0] = params
        if precision is not None:
            p.precision = precision
        if device is not None:
            p.device = device
        ctx = C.c_void_p()
        _check(lib.mms_create(C.byref(p), C.byref(ctx)), "mms_create")
        self._ctx = ctx
        self.params = p
        self.shape = tuple(x + 2 for x in p.grid)  # halo'd (x, y, z)

    # -- lifetime
    def close(self) -> None:
        if getattr(self, "_ctx", None):
            _lib().mms_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- stepping
    def step(self, nsteps: int = 1) -> None:
        _check(_lib().mms_step(self._ctx, int(nsteps)), "mms_step", self._ctx)

    def run(self, verbose: int = 0) -> None:
        _check(_lib().mms_run(self._ctx, int(verbose)), "mms_run", self._ctx)

    @property
    def timestep(self) -> int:
        v = C.c_uint64()
        _check(_lib().mms_get_timestep(self._ctx, C.byref(v)), "mms_get_timestep", self._ctx)
        return int(v.value)

    @property
    def num_grains(self) -> int:
        v = C.c_int()
        _check(_lib().mms_get_num_grains(self._ctx, C.byref(v)), "mms_get_num_grains", self._ctx)
        return int(v.value)

    @property
    def uses_tma(self) -> bool:
        return bool(_lib().mms_uses_tma(self._ctx))

    @property
    def kernel_launches(self) -> int:
        return int(_lib().mms_kernel_launches(self._ctx))

    # -- streams and timing
    def set_stream(self, cuda_stream: int | None) -> None:
        _check(_lib().mms_set_stream(self._ctx, C.c_void_p(cuda_stream or 0)), "mms_set_stream", self._ctx)

    def set_profiling(self, on: bool) -> None:
        _check(_lib().mms_set_profiling(self._ctx, int(on)), "mms_set_profiling", self._ctx)

    def set_stencil_tile(self, cells_per_thread: int, zchunk: int = 0) -> None:
        """Stencil CTA tile: (32 x cells_per_thread) x 8 cells, zchunk planes (0 = auto)."""
        _check(_lib().mms_set_stencil_tile(self._ctx, cells_per_thread, zchunk), "mms_set_stencil_tile", self._ctx)

    def stencil_tile(self) -> tuple[int, int]:
        cpt, zc = C.c_int(), C.c_int()
        _check(_lib().mms_get_stencil_tile(self._ctx, C.byref(cpt), C.byref(zc)), "mms_get_stencil_tile", self._ctx)
        return cpt.value, zc.value

    def set_am_tile(self, rows: int) -> None:
        """FP32 AM contraction tile rows: 64-128 (multiple of 16), 256, or 0 = the default (128)."""
        _check(_lib().mms_set_am_tile(self._ctx, rows), "mms_set_am_tile", self._ctx)

    def am_tile(self) -> int:
        r = C.c_int()
        _check(_lib().mms_get_am_tile(self._ctx, C.byref(r)), "mms_get_am_tile", self._ctx)
        return r.value

    def autotune(self, reps: int = 5) -> tuple[int, int, float]:
        """Picks the fastest stencil tile (state untouched); returns (cells_per_thread, zchunk, ms)."""
        cpt, zc, ms = C.c_int(), C.c_int(), C.c_double()
        _check(_lib().mms_autotune(self._ctx, reps, C.byref(cpt), C.byref(zc), C.byref(ms)), "mms_autotune",
               self._ctx)
        return cpt.value, zc.value, ms.value

    # -- frozen-CA adjoint
    def adjoint_record(self, nsteps: int, checkpoint_every: int = 100) -> None:
        """Runs nsteps steps recording the CA decisions and checkpoints."""
        _check(_lib().mms_adjoint_record(self._ctx, nsteps, checkpoint_every), "mms_adjoint_record", self._ctx)

    def _target(self, target: np.ndarray) -> np.ndarray:
        t = np.ascontiguousarray(target, dtype=np.float64)
        if t.size != self.num_cells():
            raise ValueError("target must be a halo'd field of the domain")
        return t

    def adjoint_gradient(self, target_ce: np.ndarray) -> dict:
        """Loss 1/2 sum (ce - target)^2 and its gradient w.r.t. Dliq, part_coef, GibbsThomsonCoef."""
        t = self._target(target_ce)
        r = AdjointResult()
        _check(_lib().mms_adjoint_gradient(self._ctx, t.ctypes.data, C.byref(r)), "mms_adjoint_gradient",
               self._ctx)
        return {"loss": r.loss, "Dliq": r.dL_dDliq, "part_coef": r.dL_dpart_coef, "gibbs": r.dL_dgibbs,
                "steps": int(r.steps)}

    def adjoint_replay_loss(self, target_ce: np.ndarray, scale=(1.0, 1.0, 1.0)) -> float:
        t = self._target(target_ce)
        sc = (C.c_double * 3)(*scale)
        out = C.c_double()
        _check(_lib().mms_adjoint_replay_loss(self._ctx, t.ctypes.data, sc, C.byref(out)),
               "mms_adjoint_replay_loss", self._ctx)
        return out.value

    def adjoint_release(self) -> None:
        _check(_lib().mms_adjoint_release(self._ctx), "mms_adjoint_release", self._ctx)

    def kernel_stats(self) -> dict[str, tuple[float, int]]:
        lib = _lib()
        out = {}
        for k in range(lib.mms_kernel_count()):
            ms, n = C.c_double(), C.c_uint64()
            _check(lib.mms_kernel_stats(self._ctx, k, C.byref(ms), C.byref(n)), "mms_kernel_stats", self._ctx)
            out[lib.mms_kernel_name(k).decode()] = (ms.value, int(n.value))
        return out

    # -- fields (halo'd, indexed [z, y, x] like growth.c:70)
    def num_cells(self) -> int:
        return int(_lib().mms_num_cells(self._ctx))

    def download(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """The halo'd field as [z, y, x(, component)]; `out` (contiguous, the
        field's dtype and size, e.g. a view of pinned memory) is filled instead
        of a new array."""
        f = FIELD[name]
        dt, comp = _FIELD_DTYPE[f]
        n = self.num_cells()
        if out is None:
            out = np.empty(n * comp, dtype=dt)
        elif out.dtype != dt or out.size != n * comp or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous array of the field's dtype and size")
        _check(_lib().mms_download(self._ctx, f, out.ctypes.data), f"mms_download({name})", self._ctx)
        nx, ny, nz = self.shape
        return out.reshape((nz, ny, nx, comp) if comp > 1 else (nz, ny, nx))

    def upload(self, name: str, arr: np.ndarray) -> None:
        f = FIELD[name]
        dt, comp = _FIELD_DTYPE[f]
        a = np.ascontiguousarray(arr, dtype=dt).reshape(-1)
        if a.size != self.num_cells() * comp:
            raise ValueError("field size mismatch")
        _check(_lib().mms_upload(self._ctx, f, a.ctypes.data), f"mms_upload({name})", self._ctx)

    def reduce(self, what: str = "fs_fraction") -> float:
        v = C.c_double()
        _check(_lib().mms_reduce(self._ctx, REDUCE[what], C.byref(v)), "mms_reduce", self._ctx)
        return float(v.value)

    def step_reduce(self, nsteps: int = 1, what: str = "fs_fraction") -> float:
        """step(nsteps) then reduce(what) with one synchronisation (the
        reference loop's doiteration + computeFS, loop.c:227-234)."""
        v = C.c_double()
        _check(_lib().mms_step_reduce(self._ctx, int(nsteps), REDUCE[what], C.byref(v)), "mms_step_reduce",
               self._ctx)
        return float(v.value)

    # -- sites, orientations, grains
    def set_sites(self, gxyz: np.ndarray, thresholds: np.ndarray) -> None:
        g = np.ascontiguousarray(gxyz, dtype=np.int32).reshape(-1, 3)
        t = np.ascontiguousarray(thresholds, dtype=np.float32).reshape(-1)
        _check(_lib().mms_set_sites(self._ctx, len(t), g.ctypes.data, t.ctypes.data),
               "mms_set_sites", self._ctx)

    def checkpoint_save(self, path: str) -> None:
        _check(_lib().mms_checkpoint_save(self._ctx, str(path).encode()), "mms_checkpoint_save", self._ctx)

    def checkpoint_load(self, path: str) -> None:
        _check(_lib().mms_checkpoint_load(self._ctx, str(path).encode()), "mms_checkpoint_load", self._ctx)

    def write_vtk(self, base: str | None = None) -> None:
        """<base>_<ts>.pvtu + <base>_<sbid>/<ts>.vtu (io_vtk.c layout)."""
        _check(_lib().mms_write_vtk(self._ctx, base.encode() if base else None), "mms_write_vtk", self._ctx)

    def write_xdmf(self, base: str | None = None) -> None:
        """<base>_ts.xmf + <base>_r<rank>/<ts>.raw + <base>_gbl.raw (io_xdmf.c
        layout with raw binary datasets); with RandomizeGrains this draws the
        grain renumbering from rank 0's stream as the reference does."""
        _check(_lib().mms_write_xdmf(self._ctx, base.encode() if base else None), "mms_write_xdmf", self._ctx)

    def xdmf_renumbering(self) -> np.ndarray:
        n = C.c_int()
        _check(_lib().mms_xdmf_renumbering(self._ctx, 0, None, C.byref(n)), "mms_xdmf_renumbering", self._ctx)
        out = np.empty(n.value, dtype=np.uint64)
        _check(_lib().mms_xdmf_renumbering(self._ctx, n.value, out.ctypes.data, C.byref(n)), "mms_xdmf_renumbering",
               self._ctx)
        return out

    def test_hold_list_block(self, block: int, polls: int = 0) -> None:
        """Failure-detection test hook (mms_test_hold_list_block): from the
        next step on, list block `block` publishes no status word and the
        look-back waits give up after `polls` polls (-1: off)."""
        _check(_lib().mms_test_hold_list_block(self._ctx, block, polls), "mms_test_hold_list_block", self._ctx)

    def set_grains(self, rotmats: np.ndarray) -> None:
        """Grains 1..n of a pre-filled microstructure (row-major 3x3 rotations)."""
        r = np.ascontiguousarray(rotmats, dtype=np.float64).reshape(-1, 9)
        _check(_lib().mms_set_grains(self._ctx, len(r), r.ctypes.data), "mms_set_grains", self._ctx)

    def set_site_orientations(self, gxyz: np.ndarray, rotmats: np.ndarray) -> None:
        g = np.ascontiguousarray(gxyz, dtype=np.int32).reshape(-1, 3)
        r = np.ascontiguousarray(rotmats, dtype=np.float64).reshape(-1, 9)
        _check(_lib().mms_set_site_orientations(self._ctx, len(r), g.ctypes.data, r.ctypes.data),
               "mms_set_site_orientations", self._ctx)

    def grains(self) -> list[Grain]:
        n = self.num_grains
        arr = (Grain * n)()
        _check(_lib().mms_get_grains(self._ctx, 0, n, arr), "mms_get_grains", self._ctx)
        return list(arr)

    def grain_summary(self, csv_path: str | None = None) -> GrainSummary:
        s = GrainSummary()
        path = csv_path.encode() if csv_path else None
        _check(_lib().mms_output_grains(self._ctx, path, C.byref(s)), "mms_output_grains", self._ctx)
        return s


class _BatchDomain(Domain):
    """A domain owned by a Batch: fields, reductions and grains, no stepping."""

    def __init__(self, batch: "Batch", ctx, params: Params):
        self._ctx = ctx
        self._batch = batch
        self.params = params
        self.shape = tuple(x + 2 for x in params.grid)

    def close(self) -> None:  # owned by the batch
        self._ctx = None

    def step(self, n: int = 1) -> None:
        raise MmsError(10, "step", "a batched domain steps with its Batch")


class Batch:
    """Many independent domains stepped together (mms_batch_*): one CUDA graph
    per step with a single persistent stencil launch over all domains."""

    def __init__(self, params: list, precision: int = PREC_F64, device: int = 0):
        arr = (Params * len(params))()
        for i, p in enumerate(params):
            C.memmove(C.byref(arr[i]), C.byref(p), C.sizeof(Params))
            arr[i].precision = precision
            arr[i].device = device
        h = C.c_void_p()
        _check(_lib().mms_batch_create(len(params), arr, C.byref(h)), "mms_batch_create")
        self._b = h
        self.domains = [_BatchDomain(self, C.c_void_p(_lib().mms_batch_domain(h, i)), arr[i])
                        for i in range(len(params))]

    def __len__(self) -> int:
        return len(self.domains)

    def _chk(self, st: int, where: str) -> None:
        if st != 0:
            raise MmsError(st, where, (_lib().mms_batch_last_error(self._b) or b"").decode())

    def step(self, n: int = 1) -> None:
        self._chk(_lib().mms_batch_step(self._b, n), "mms_batch_step")

    def set_stencil_tile(self, cells_per_thread: int, zchunk: int = 0) -> None:
        self._chk(_lib().mms_batch_set_stencil_tile(self._b, cells_per_thread, zchunk), "mms_batch_set_stencil_tile")

    def stencil_tile(self) -> tuple[int, int, int]:
        c, z, g = C.c_int(), C.c_int(), C.c_int()
        self._chk(_lib().mms_batch_get_stencil_tile(self._b, C.byref(c), C.byref(z), C.byref(g)),
                  "mms_batch_get_stencil_tile")
        return c.value, z.value, g.value

    def autotune(self, reps: int = 3) -> tuple[int, int, float]:
        c, z, ms = C.c_int(), C.c_int(), C.c_double()
        self._chk(_lib().mms_batch_autotune(self._b, reps, C.byref(c), C.byref(z), C.byref(ms)), "mms_batch_autotune")
        return c.value, z.value, ms.value

    @property
    def kernel_launches(self) -> int:
        return int(_lib().mms_batch_kernel_launches(self._b))

    def close(self) -> None:
        if self._b:
            for d in self.domains:
                d.close()
            _lib().mms_batch_destroy(self._b)
            self._b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------ one domain split into z-slabs
def slab_layout(params: Params, nslabs: int, slab: int) -> SlabLayout:
    """Which whole-domain z cells and emulated ranks slab `slab` of `nslabs`
    owns (no device needed)."""
    out = SlabLayout()
    _check(_lib().mms_slab_layout_of(C.byref(params), nslabs, slab, C.byref(out)), "mms_slab_layout_of")
    return out


class SlabDomain(Domain):
    """One z-slab of a domain split over devices (mms_slab_create): whole
    layers of subblocks, with a one-plane halo that the step's two exchanges
    fill from the neighbouring slabs.  Fields, downloads and reductions are
    the slab's own; grain records cover the whole domain."""

    def __init__(self, params: Params, nslabs: int, slab: int, precision: int | None = None,
                 device: int | None = None):
        lib = _lib()
        p = Params()
        C.pointer(p)[0] = params
        if precision is not None:
            p.precision = precision
        if device is not None:
            p.device = device
        ctx = C.c_void_p()
        _check(lib.mms_slab_create(C.byref(p), nslabs, slab, C.byref(ctx)), "mms_slab_create")
        self._ctx = ctx
        self.global_params = p
        self.layout = SlabLayout()
        _check(lib.mms_slab_get_layout(ctx, C.byref(self.layout)), "mms_slab_get_layout", ctx)
        sp = Params()
        C.pointer(sp)[0] = p
        sp.gnsbz = self.layout.z_cells // p.gsdimz
        self.params = sp
        self.shape = tuple(x + 2 for x in sp.grid)

    def step(self, nsteps: int = 1) -> None:
        if self.layout.nslabs == 1:
            super().step(nsteps)
        else:
            raise MmsError(1, "step", "a slab steps with its group (SlabGroup, or launch/exchange per phase)")

    # -- caller-driven stepping (one process per device)
    def launch(self, phase: int, resume: bool = False) -> None:
        _check(_lib().mms_slab_launch(self._ctx, phase, int(resume)), "mms_slab_launch", self._ctx)

    def exchange_plan(self, point: int, timestep: int) -> list[tuple[int, int, int, int, int]]:
        """(kind, peer, send pointer, recv pointer, bytes) of exchange point
        0 or 1 of the step that starts at `timestep`."""
        n = C.c_int()
        buf = (SlabXfer * 32)()
        _check(_lib().mms_slab_exchange_plan(self._ctx, point, timestep, buf, 32, C.byref(n)),
               "mms_slab_exchange_plan", self._ctx)
        return [(x.kind, x.peer, int(x.send or 0), int(x.recv or 0), int(x.bytes)) for x in buf[:n.value]]

    def poll(self) -> tuple[int, bool]:
        """(timestep, stalled for want of pre-drawn orientations)."""
        t, s = C.c_uint64(), C.c_int()
        _check(_lib().mms_slab_poll(self._ctx, C.byref(t), C.byref(s)), "mms_slab_poll", self._ctx)
        return int(t.value), bool(s.value)

    def refill(self) -> None:
        _check(_lib().mms_slab_refill(self._ctx), "mms_slab_refill", self._ctx)


class SlabGroup:
    """All slabs of one domain in this process (mms_slab_group_step): each on
    devices[s % len(devices)], exchanges as device (peer) copies."""

    def __init__(self, params: Params, nslabs: int, precision: int = PREC_F64, devices=(0,)):
        self.slabs = [SlabDomain(params, nslabs, s, precision, devices[s % len(devices)])
                      for s in range(nslabs)]
        self.params = self.slabs[0].global_params
        self._arr = (C.c_void_p * nslabs)(*[d._ctx.value for d in self.slabs])

    def __len__(self) -> int:
        return len(self.slabs)

    def step(self, n: int = 1) -> None:
        st = _lib().mms_slab_group_step(self._arr, len(self.slabs), int(n))
        if st != 0:
            detail = "; ".join(filter(None, ((_lib().mms_last_error(d._ctx) or b"").decode() for d in self.slabs)))
            raise MmsError(st, "mms_slab_group_step", detail)

    @property
    def timestep(self) -> int:
        return self.slabs[0].timestep

    @property
    def num_grains(self) -> int:
        return self.slabs[0].num_grains

    def download(self, name: str) -> np.ndarray:
        """The whole domain's halo'd field [z, y, x(, c)], assembled from the
        slabs' interior planes (the outer halo planes from the end slabs)."""
        parts = [d.download(name) for d in self.slabs]
        planes = [parts[0][:1]] + [q[1:-1] for q in parts] + [parts[-1][-1:]]
        return np.concatenate(planes, axis=0)

    def reduce(self, what: str = "fs_fraction") -> float:
        """Sums over the slabs (the reference's MPI_Allreduce order differs
        from one domain's, as here)."""
        if what == "fs_fraction":
            nx, ny, nz = self.params.grid
            v = sum(d.reduce("solid_volume") for d in self.slabs)
            return v / (nx * ny * nz * self.params.cellSize ** 3)
        return sum(d.reduce(what) for d in self.slabs)

    def grains(self) -> list[Grain]:
        return self.slabs[0].grains()

    def set_sites(self, gxyz: np.ndarray, thresholds: np.ndarray) -> None:
        for d in self.slabs:
            d.set_sites(gxyz, thresholds)

    def set_site_orientations(self, gxyz: np.ndarray, rotmats: np.ndarray) -> None:
        for d in self.slabs:
            d.set_site_orientations(gxyz, rotmats)

    def set_grains(self, rotmats: np.ndarray) -> None:
        for d in self.slabs:
            d.set_grains(rotmats)

    def upload(self, name: str, arr: np.ndarray) -> None:
        """Uploads the whole domain's halo'd field [z, y, x(, c)] slab by slab."""
        a = np.asarray(arr)
        for d in self.slabs:
            z0 = d.layout.z_begin
            d.upload(name, a[z0:z0 + d.layout.z_cells + 2])

    @property
    def kernel_launches(self) -> int:
        return sum(d.kernel_launches for d in self.slabs)

    def close(self) -> None:
        for d in self.slabs:
            d.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
