#!/usr/bin/env python3
"""Throughput of the muMatScale CA step on B200: cell-updates/s.

Default workload (the driver's line): the AM single-track melt pool, 512 x
256 x 128 cells, dx = 1 um, binary Al-Cu (C0 = 4.5 wt%, m = -2.6 K/wt%, k =
0.14, D_l = 3e-9, D_s = 3e-13 m^2/s), the reference's moving-source
quadrature temperature (AnalyticalThermal 1, temperature.c:62-123) at 0.5
m/s, 150 W, absorptivity 0.4, k_th = 100 W/m/K, alpha = 3e-5 m^2/s; a
substrate of columnar grains (mean width 20 um, random orientations) in
interior planes 1..120; bulk sites at 1e14 m^-3 with undercooling N(3 K,
1 K).  The deck is split into the same NSubblocks as the reference arm
uses, so both arms draw the same sites from the same per-rank streams.  A
"step" is one timestep (doiteration) of the whole domain; the metric counts
interior cells x steps / second.

GPU arm: ``value`` is the FP32 form (FP32 ce/cl/fs, tensor-core
temperature, FP64 octahedra, thresholds and reductions); the FP64 plain form
is reported beside it, with the FP32 form's error against it after the
timed steps (grain-id mismatch fraction, relative L2 of ce, max |fs error|,
max |T error| / max T).  Timing: W untimed steps, then K steps bracketed by
CUDA events on the stream the library launches on, synchronised on both
sides; the fields (about 0.7 GB in FP32, 1.1 GB in FP64) are larger than
the 126 MB L2, so no flush is needed.  ``e2e``: the same K steps through the
public API from a fresh context, with the substrate uploaded from pinned
host memory, the fraction solid read back every step and the grain ids and
ce read back at the end, all inside the timed region.  Under torchrun every
rank runs its own replica (weak scaling; --workload slabs splits one
domain) and the maximum over ranks is taken.  The multi-grain
directional-solidification deck (256^3) is reported under ``cfg2``.

Reference arm (--impl reference): the unmodified reference compiled from
its sources (oracle/_ref/mmsref), run as MPI ranks over the host cores
through the project's shared-memory MPI shim on the same deck and
substrate, timing K steps after W steps from per-step timestamps.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s, FP32 form vs FP64 plain (1 B200); stencil HBM GB/s vs peak"
UNIT = "cell-updates/s"
N_CELL = 256
# Al-Cu alloy: liquidus = 933.47 - 2.6*4.5 (pure-Al melting point assumed);
# solidus = 933.47 - 2.6*4.5/0.14
T_LIQ = 933.47 - 2.6 * 4.5
T_SOL = 933.47 - 2.6 * 4.5 / 0.14
DX = 2e-6
# D_l dt/dx^2 = 0.04.  With k = 0.14 the reference's explicit update keeps
# ce >= 0 only while 3 D_l dt/dx^2 < k (a solid cell, cl = ce/k, next to six
# liquid cells); at 0.15 and at 0.10 the reference itself aborts on this deck
# (ce < 0, growth.c:163-165) within ~75 steps.
DT = 0.04 * DX * DX / 3e-9
# algorithmic bytes per cell of the dominant kernel k_diffuse_fs:
# read ce, cl, fs + write ce, cl, fs + read gr
BYTES_DIFFUSE = {"f64": 3 * 8 * 2 + 4, "f32": 3 * 4 * 2 + 4}
# full-step dense bytes per cell-update (ce, cl, fs read+write, gr, threshold)
BYTES_STEP = {"f64": 56, "f32": 32}
# the AM deck's stencil also reads the temperature field (FP64 in the FP64
# form, FP32 in the FP32 form)
BYTES_DIFFUSE_AM = {"f64": BYTES_DIFFUSE["f64"] + 8, "f32": BYTES_DIFFUSE["f32"] + 4}

# AM melt-pool deck (the default workload)
AM_DIMS = (512, 256, 128)
AM_DX = 1e-6
AM_TOP = AM_DIMS[2] - 8        # substrate: interior planes 1..120
AM_SUB_WIDTH, AM_SUB_SEED = 20e-6, 11
AM_DT = 0.04 * AM_DX * AM_DX / 3e-9


def deck_text(nsb=(1, 1, 1), n=N_CELL, seed=20261203) -> str:
    sb = [n // nsb[0], n // nsb[1], n // nsb[2]]
    return f"""BaseFileName bench256
NSubblocks {nsb[0]} {nsb[1]} {nsb[2]}
NCellsPerSB {sb[0]} {sb[1]} {sb[2]}
FaceCtrl 1 1 1 1 1 1
CellSize {DX!r}
FSGrow 0.66
TimeStep {DT!r}
RandSeedVal {seed}
TipCurvature 0
GibbsThomsonCoef 2.4e-7
FinishTime 0
FsFinish 1.1
LiquidusTemp {T_LIQ!r}
SolidusTemp {T_SOL!r}
Cinit 4.5
m_solute0 0 0 -2.6
part_coef0 0 0 0.14
Dsol 3e-13
Dliq 3e-9
InitialTemperature {T_LIQ - 2.5!r}
Gradient 1e4
Velocity 1e-3
CoolingRate 0
ScreenPFreq 0
MaxGrainDensity 1e13
GNGaussCentre 2.0
GNGaussSigma 0.5
MaxGrainDensitySurf 1e10
GNGaussCentreSurf 2.0
GNGaussSigmaSurf 0.5
MaxTotGrains 1000000
GNOriented 1
"""


def am_deck_text(nsb=(1, 1, 1)) -> str:
    """The AM melt-pool deck split into nsb subblocks (emulated ranks)."""
    from mumatscale_b200 import workloads as W
    assert all(AM_DIMS[i] % nsb[i] == 0 for i in range(3)), nsb
    sb = [AM_DIMS[i] // nsb[i] for i in range(3)]
    d = W.am_track(AM_DIMS, AM_DX)
    d = d.replace("NSubblocks 1 1 1", f"NSubblocks {nsb[0]} {nsb[1]} {nsb[2]}")
    return d.replace(f"NCellsPerSB {AM_DIMS[0]} {AM_DIMS[1]} {AM_DIMS[2]}", f"NCellsPerSB {sb[0]} {sb[1]} {sb[2]}")


def am_substrate():
    """The columnar substrate of the AM deck: (column grain ids, rotations)."""
    from mumatscale_b200 import workloads as W
    return W.columnar_columns(AM_DIMS[0], AM_DIMS[1], AM_DX, AM_SUB_WIDTH, AM_SUB_SEED)


def am_host_fields(cols, gr=None, fs=None):
    """gr and fs of the substrate in the halo'd layout (into gr / fs when
    given, e.g. pinned buffers): ids in planes 1..AM_TOP, fs = 1 there."""
    shape = (AM_DIMS[2] + 2, AM_DIMS[1] + 2, AM_DIMS[0] + 2)
    import numpy as np
    gr = np.zeros(shape, dtype=np.int32) if gr is None else gr.reshape(shape)
    fs = np.zeros(shape, dtype=np.float64) if fs is None else fs.reshape(shape)
    gr[...] = 0
    gr[1:AM_TOP + 1, 1:-1, 1:-1] = cols[None]
    fs[...] = 0.0
    fs[gr > 0] = 1.0
    return gr, fs


def am_fill(dom, rot, gr, fs) -> None:
    """The substrate into a fresh context: grains 1..n, then gr and fs."""
    dom.set_grains(rot)
    dom.upload("gr", gr)
    dom.upload("fs", fs)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML read from a thread every 2 ms and once more as the region
    ends (the device found by its PCI bus id), else nvidia-smi every 100 ms.
    Reads only; changes nothing."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []
        self.nvml = None
        self.samples: list[tuple[float, float, set]] = []  # (sm MHz, max MHz, reasons)
        self._stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        import torch
        pr = torch.cuda.get_device_properties(self.gpu)
        try:
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            pass
        try:
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(pr.uuid))
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def _sample(self):
        nv, h = self.nvml
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        try:
            sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append((sm, self._max, {k for k, b in bits.items() if r & b}))
        except Exception:
            pass

    def _poll(self):
        while not self._stop.is_set():
            self._sample()
            self._stop.wait(0.002)

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            nv, h = self.nvml
            self._max = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._t = threading.Thread(target=self._poll, daemon=True)
            self._t.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        # one reading taken here, as the timed region ends, so that a region
        # shorter than the polling thread's first wake-up still has one
        if self.nvml:
            self._sample()
        self._stop.set()
        if self.nvml:
            self._t.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        for s, m, r in self.samples:
            sm.append(s)
            mx = m
            reasons |= r
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.samples else "nvidia-smi"}


# --------------------------------------------------------------- helpers
def dist_env():
    from mumatscale_b200.distributed import dist_env as env
    return env()


def measured_peak_gbs() -> tuple[float, str]:
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return float(json.loads(f.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def measured_peak_tflops() -> float:
    """Dense bf16 GEMM peak (burst) of MEASURED_PEAKS.json, else the fallback."""
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return float(json.loads(f.read_text())["bf16_tflops"])
        except Exception:
            pass
    return 1590.0


def ncu_traffic_per_cell(dtype: str, workload: str = "ds256"):
    """DRAM bytes per cell of one stencil launch from a committed ncu summary
    (profiles/k_diffuse_fs_traffic.json: keys "f64"/"f32" for the 256^3
    directional deck, "am_f64"/"am_f32" for the AM deck), or None."""
    f = ROOT / "profiles" / "k_diffuse_fs_traffic.json"
    key = dtype if workload == "ds256" else f"{workload}_{dtype}"
    if f.exists():
        try:
            d = json.loads(f.read_text())
            return d[key]["dram_bytes_per_cell"]
        except Exception:
            return None
    return None


def ref_procs(cores: int) -> tuple[int, tuple[int, int, int]]:
    """Largest power of two <= min(cores, 64), split over z, y, x."""
    n = 1
    while n * 2 <= min(cores, 64):
        n *= 2
    nsb = [1, 1, 1]
    k, ax = n, 2
    while k > 1:
        nsb[ax] *= 2
        k //= 2
        ax = (ax - 1) % 3
    return n, (nsb[0], nsb[1], nsb[2])


def run_reference(workload: str, nsteps_w: int, nsteps_k: int, cores: int | None = None,
                  timeout: float = 1800):
    """Times the unmodified reference (oracle/_ref/mmsref) on a bench deck:
    workload "am" (the default AM melt pool with its substrate, injected
    through MMSREF_INJECT_SUBSTRATE) or "ds256" (directional solidification).
    Returns (result, None) or (None, why)."""
    ref = ROOT / "oracle" / "_ref" / "mmsref"
    if not ref.exists():
        return None, "oracle/_ref/mmsref not built"
    cores = cores or (os.cpu_count() or 1)
    nproc, nsb = ref_procs(cores)
    with tempfile.TemporaryDirectory() as td:
        deck = Path(td) / "bench.in"
        env = dict(os.environ, MMSREF_NP=str(nproc), OMP_NUM_THREADS="1")
        if workload == "am":
            from mumatscale_b200 import workloads as W
            text = am_deck_text(nsb).replace("FinishTime 0\n",
                                             f"FinishTime {(nsteps_w + nsteps_k - 0.5) * AM_DT!r}\n")
            cols, rot = am_substrate()
            W.write_substrate_file(Path(td) / "substrate.bin", cols, rot, AM_TOP)
            env["MMSREF_INJECT_SUBSTRATE"] = str(Path(td) / "substrate.bin")
            cells = AM_DIMS[0] * AM_DIMS[1] * AM_DIMS[2]
        else:
            text = deck_text(nsb).replace("FinishTime 0", f"FinishTime {(nsteps_w + nsteps_k - 0.5) * DT!r}")
            cells = N_CELL ** 3
        deck.write_text(text)
        times = Path(td) / "times.txt"
        env["MMSREF_STEP_TIMES"] = str(times)
        t0 = time.time()
        try:
            r = subprocess.run([str(ref), "-c", str(deck)], cwd=td, env=env, capture_output=True, text=True,
                               timeout=timeout)
        except subprocess.TimeoutExpired:
            return None, f"reference did not finish within {timeout:.0f} s"
        wall = time.time() - t0
        if r.returncode != 0:
            return None, f"reference exited {r.returncode}: {r.stderr[-300:]}"
        ts = {}
        for line in times.read_text().split("\n"):
            if line.strip():
                a, b = line.split()
                ts[int(a)] = float(b)
        t_start = ts.get(nsteps_w)
        t_end = ts.get(nsteps_w + nsteps_k)
        if t_start is None or t_end is None:
            return None, "reference step timestamps missing"
        grains = None
        for line in r.stdout.splitlines():
            w = line.split()
            if len(w) > 1 and w[1] == "grains.":
                grains = int(w[0])  # output_grains: num_grains - 1 (grain.c:823)
        sec = t_end - t_start
        return {"value": cells * nsteps_k / sec, "sec": sec, "procs": nproc, "nsubblocks": nsb,
                "wall": wall, "steps": nsteps_k, "grains": grains, "cells": cells}, None


# ---------------------------------------------------------------- GPU arm
def ds256_workload(args) -> None:
    """The multi-grain directional-solidification deck (256^3) as its own
    line: FP64 plain form as value, FP32 beside it, e2e, CPU baseline."""
    import numpy as np
    import torch
    import mumatscale_b200 as M

    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    stream = torch.cuda.current_stream()

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    K, W = args.steps, args.warmup
    cells = N_CELL ** 3
    td = tempfile.mkdtemp()
    deck = Path(td) / "bench.in"
    deck.write_text(deck_text())
    params = M.read_deck(deck)
    out: dict = {}
    launches_total = 0
    for form, prec in (("f64", M.PREC_F64), ("f32", M.PREC_F32)):
        dom = M.Domain(params, precision=prec, device=dev)
        dom.set_stream(stream.cuda_stream)
        tile = dom.autotune(reps=5)  # stencil tile for this grid and form
        dom.step(W)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = dom.kernel_launches
        with ClockSampler(dev) as clk:
            e0.record(stream)
            dom.step(K)
            e1.record(stream)
            torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1))
        launches = dom.kernel_launches - l0
        launches_total += launches
        # per-kernel device time over a second timed pass of K steps
        dom.set_profiling(True)
        dom.step(K)
        torch.cuda.synchronize()
        ks = dom.kernel_stats()
        dom.set_profiling(False)
        out[form] = {"ms_total": ms, "launches": launches, "kernels": ks, "clocks": clk.summary(),
                     "tile": {"cells_per_thread": tile[0], "zchunk": tile[1], "cta_cells": [32 * tile[0], 8]},
                     "grains": dom.num_grains, "timestep": dom.timestep}
        if form == "f64":
            # end to end through the public API with host buffers: upload the
            # whole state from pinned host memory, K steps each followed by a
            # device->host read of the fraction solid (loop.c's screen value,
            # one mms_step_reduce call per step), and a final download of
            # grain ids and ce
            n = dom.num_cells()
            host = {f: torch.empty(n * (3 if f == "dc" else 1),
                                   dtype=torch.int32 if f == "gr" else torch.float64).pin_memory()
                    for f in ("ce", "cl", "fs", "gr", "dc")}
            for f, t in host.items():
                arr = dom.download(f).reshape(-1)
                t.numpy()[:] = arr
            host_out = {f: torch.empty(n, dtype=torch.int32 if f == "gr" else torch.float64).pin_memory()
                        for f in ("gr", "ce")}
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            h2d = 0
            for f, t in host.items():
                dom.upload(f, t.numpy())
                h2d += t.numel() * t.element_size()
            d2h = 0
            for _ in range(K):
                dom.step_reduce(1, "fs_fraction")
                d2h += 8
            gr = dom.download("gr", out=host_out["gr"].numpy())
            ce = dom.download("ce", out=host_out["ce"].numpy())
            d2h += gr.nbytes + ce.nbytes
            torch.cuda.synchronize()
            e2e_s = max_over_ranks(time.perf_counter() - t0)
            out["e2e"] = {"value": ws * cells * K / e2e_s, "unit": UNIT,
                          "h2d_bytes_per_step": h2d // K, "d2h_bytes_per_step": d2h // K}
        dom.close()
        del dom

    if rank != 0:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    f64, f32 = out["f64"], out["f32"]
    value = ws * cells * K / (f64["ms_total"] / 1e3)
    value32 = ws * cells * K / (f32["ms_total"] / 1e3)
    peak, peak_kind = measured_peak_gbs()
    kms, kn = f64["kernels"]["k_diffuse_fs"]
    per_launch_s = kms / 1e3 / max(kn, 1)
    achieved = BYTES_DIFFUSE["f64"] * cells / per_launch_s / 1e9
    kms32, kn32 = f32["kernels"]["k_diffuse_fs"]
    achieved32 = BYTES_DIFFUSE["f32"] * cells / (kms32 / 1e3 / max(kn32, 1)) / 1e9
    tr = ncu_traffic_per_cell("f64")
    step_ms = f64["ms_total"] / K
    share = {k: round(v[0] / max(1e-9, sum(x[0] for x in f64["kernels"].values())), 4)
             for k, v in f64["kernels"].items() if v[1]}
    cpu = None
    if not args.no_cpu_baseline:
        res, why = run_reference("ds256", 2, args.cpu_steps)
        if res:
            cpu = {"value": res["value"], "unit": UNIT, "cores": res["procs"], "kind": "reference",
                   "sample": f"{res['steps']} timesteps of the same 256^3 deck after 2 warm-up steps, "
                             f"{res['procs']} MPI ranks (NSubblocks {res['nsubblocks']}) of the reference "
                             f"through the shared-memory MPI shim, {res['sec']:.2f} s"}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": why}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "multi-grain directional solidification, 256^3 cells, FP64 plain form",
                   "cells": cells, "dx_m": DX, "dt_s": DT, "G_K_per_m": 1e4, "V_m_per_s": 1e-3,
                   "parallelism": f"replicas x{ws}", "l2": "inputs larger than L2 (about 1.1 GB of fields)",
                   "grains_after_run": f64["grains"], "stencil_tile": f64["tile"]},
        "fp32_form": {"value": value32, "ms_per_step": f32["ms_total"] / K, "ratio_vs_fp64": value32 / value,
                      "k_diffuse_fs_gbs": achieved32, "k_diffuse_fs_frac": achieved32 / peak,
                      "stencil_tile": f32["tile"]},
        "roofline": {"bound": "hbm", "kernel": "k_diffuse_fs", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_cell": BYTES_DIFFUSE["f64"],
                     "traffic": (tr * cells) if tr else None,
                     "kernel_ms_per_launch": per_launch_s * 1e3},
        "kernel_share": share,
        "e2e": out["e2e"],
        "gpu_launches": f64["launches"],
        "clocks": f64["clocks"],
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _errors(d32, d64) -> dict:
    """The FP32 form against the FP64 plain form, interior cells: grain-id
    mismatch fraction, relative L2 of ce, max |fs error|, max |T error| over
    max |T| (all cells)."""
    import numpy as np

    def inner(x):
        return x[1:-1, 1:-1, 1:-1]
    g32, g64 = inner(d32.download("gr")), inner(d64.download("gr"))
    c32, c64 = inner(d32.download("ce")), inner(d64.download("ce"))
    f32, f64 = inner(d32.download("fs")), inner(d64.download("fs"))
    t32, t64 = d32.download("temperature"), d64.download("temperature")
    return {"grain_id_mismatch": float((g32 != g64).mean()),
            "ce_rel_l2": float(np.linalg.norm(c32 - c64) / np.linalg.norm(c64)),
            "fs_max_abs": float(np.abs(f32 - f64).max()),
            "T_max_rel": float(np.abs(t32 - t64).max() / max(np.abs(t64).max(), 1e-300)),
            "at_step": d64.timestep}


def _dist(ws):
    import torch
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(dist_env()[2])
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return barrier, max_over_ranks


def _roofline(ks: dict, steps: int, cells: int, form: str, peaks: dict) -> dict:
    """Roofline of the kernel with the largest device time in ks
    (name -> (ms over `steps` steps, launches))."""
    name = max(ks, key=lambda k: ks[k][0])
    ms, n = ks[name]
    per_launch = ms / 1e3 / max(n, 1)
    if name == "k_temp_am":
        # tables + contraction per step: 2 x 400 multiply-adds per cell the
        # step computes (x = 1..gx of every halo'd (y, z) row; the halo
        # columns are filled only where read).  Algorithmic: the FP32 form
        # issues three FP16 products per multiply-add (head x head, head x
        # remainder, remainder x head) at the dense FP16/bf16 rate, so its
        # tensor-core bound is peak / 3 in these units
        cells_t = AM_DIMS[0] * (AM_DIMS[1] + 2) * (AM_DIMS[2] + 2)
        flops = 2.0 * 400 * cells_t
        ach = flops / per_launch / 1e12
        pk = peaks["bf16_tflops"]
        return {"bound": "tensor", "kernel": name, "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                "frac": ach / pk, "frac_of_split_bound": ach / (pk / 3.0),
                "peak_source": peaks["source"] + " (dense bf16 GEMM)",
                "algorithmic_flops_per_launch": flops, "traffic": None,
                "kernel_ms_per_launch": per_launch * 1e3}
    b = BYTES_DIFFUSE_AM[form] if name == "k_diffuse_fs" else BYTES_STEP[form]
    ach = b * cells / per_launch / 1e9
    tr = ncu_traffic_per_cell(form, "am")
    return {"bound": "hbm", "kernel": name, "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": ach / peaks["hbm_gbs"], "peak_source": peaks["source"],
            "algorithmic_bytes_per_cell": b, "traffic": (tr * cells) if tr else None,
            "kernel_ms_per_launch": per_launch * 1e3}


def gpu_arm(args) -> None:
    """The default line: the AM melt-pool deck, FP32 form as value."""
    import numpy as np
    import torch
    import mumatscale_b200 as M

    ws, rank, _ = dist_env()
    barrier, max_over_ranks = _dist(ws)
    dev = torch.cuda.current_device()
    stream = torch.cuda.current_stream()
    K, Wm = args.steps, args.warmup
    cells = AM_DIMS[0] * AM_DIMS[1] * AM_DIMS[2]
    nproc, nsb = ref_procs(os.cpu_count() or 1)
    td = tempfile.mkdtemp()
    deck = Path(td) / "am.in"
    deck.write_text(am_deck_text(nsb))
    params = M.read_deck(deck)
    cols, rot = am_substrate()
    gr0, fs0 = am_host_fields(cols)
    doms, out = {}, {}
    for form, prec in (("f32", M.PREC_F32), ("f64", M.PREC_F64)):
        dom = M.Domain(params, precision=prec, device=dev)
        dom.set_stream(stream.cuda_stream)
        am_fill(dom, rot, gr0, fs0)
        tile = dom.autotune(reps=3)
        dom.step(Wm)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = dom.kernel_launches
        with ClockSampler(dev) as clk:
            e0.record(stream)
            dom.step(K)
            e1.record(stream)
            torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1))
        out[form] = {"ms_total": ms, "launches": dom.kernel_launches - l0, "clocks": clk.summary(),
                     "tile": {"cells_per_thread": tile[0], "zchunk": tile[1], "cta_cells": [32 * tile[0], 8]},
                     "grains": dom.num_grains - 1}
        if form == "f32":
            out[form]["tile"]["am_rows"] = dom.am_tile()
        doms[form] = dom
    errors = _errors(doms["f32"], doms["f64"])
    for form, dom in doms.items():
        # per-kernel device time over a second pass of K steps
        dom.set_profiling(True)
        dom.step(K)
        torch.cuda.synchronize()
        out[form]["kernels"] = dom.kernel_stats()
        dom.set_profiling(False)
        dom.close()
    del doms

    # end to end through the public API, FP32 form: a fresh context (created
    # before the clock starts), then the substrate uploaded from pinned host
    # memory, K steps each followed by a device->host read of the fraction
    # solid (loop.c's screen value), and the grain ids and ce read back
    n = (AM_DIMS[0] + 2) * (AM_DIMS[1] + 2) * (AM_DIMS[2] + 2)
    h_gr = torch.empty(n, dtype=torch.int32).pin_memory()
    h_fs = torch.empty(n, dtype=torch.float64).pin_memory()
    am_host_fields(cols, h_gr.numpy(), h_fs.numpy())
    o_gr = torch.empty(n, dtype=torch.int32).pin_memory()
    o_ce = torch.empty(n, dtype=torch.float64).pin_memory()
    with M.Domain(params, precision=M.PREC_F32, device=dev) as dom:
        dom.set_stream(stream.cuda_stream)
        # the tiles the tuner picked for this deck above
        dom.set_stencil_tile(out["f32"]["tile"]["cells_per_thread"], out["f32"]["tile"]["zchunk"])
        dom.set_am_tile(out["f32"]["tile"]["am_rows"])
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        am_fill(dom, rot, h_gr.numpy(), h_fs.numpy())
        h2d = rot.nbytes + h_gr.numel() * 4 + h_fs.numel() * 8
        d2h = 0
        for _ in range(K):
            dom.step_reduce(1, "fs_fraction")
            d2h += 8
        dom.download("gr", out=o_gr.numpy())
        dom.download("ce", out=o_ce.numpy())
        d2h += o_gr.numel() * 4 + o_ce.numel() * 8
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": ws * cells * K / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d // K,
           "d2h_bytes_per_step": d2h // K}

    cfg2 = None if args.no_cfg2 else ds256_device(args, ws, stream, barrier, max_over_ranks)

    if rank != 0:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    f32, f64 = out["f32"], out["f64"]
    value = ws * cells * K / (f32["ms_total"] / 1e3)
    value64 = ws * cells * K / (f64["ms_total"] / 1e3)
    peak, peak_kind = measured_peak_gbs()
    peaks = {"hbm_gbs": peak, "bf16_tflops": measured_peak_tflops(), "source": peak_kind}
    roof = _roofline(f32["kernels"], K, cells, "f32", peaks)
    kms, kn = f32["kernels"]["k_diffuse_fs"]
    st32 = BYTES_DIFFUSE_AM["f32"] * cells / (kms / 1e3 / max(kn, 1)) / 1e9
    kms64, kn64 = f64["kernels"]["k_diffuse_fs"]
    st64 = BYTES_DIFFUSE_AM["f64"] * cells / (kms64 / 1e3 / max(kn64, 1)) / 1e9

    def per_step(ks):
        return {k: round(v[0] / K, 5) for k, v in ks.items() if v[1]}
    cpu = None
    check = None
    if not args.no_cpu_baseline:
        w1, k1 = 1, args.cpu_steps if args.cpu_steps != 200 else 2
        res, why = run_reference("am", w1, k1)
        if res:
            cpu = {"value": res["value"], "unit": UNIT, "cores": res["procs"], "kind": "reference",
                   "sample": f"{res['steps']} timesteps of the same 512x256x128 AM deck and substrate after "
                             f"{w1} warm-up step, {res['procs']} MPI ranks (NSubblocks {res['nsubblocks']}) of "
                             f"the reference through the shared-memory MPI shim, {res['sec']:.2f} s"}
            # the same number of steps on the device, FP64 plain form: grain counts agree
            with M.Domain(params, precision=M.PREC_F64, device=dev) as d:
                am_fill(d, rot, gr0, fs0)
                d.step(w1 + k1)
                check = {"steps": w1 + k1, "reference_grains": res["grains"], "fp64_grains": d.num_grains - 1}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": why}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": Wm,
        "ms_per_step": f32["ms_total"] / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": am_config(nsb, f32["grains"]),
        "parallelism": f"replicas x{ws}",
        "fp64_plain": {"value": value64, "ms_per_step": f64["ms_total"] / K, "grains_after_run": f64["grains"],
                       "k_diffuse_fs_gbs": st64, "k_diffuse_fs_frac": st64 / peak,
                       "kernel_ms_per_step": per_step(f64["kernels"]), "stencil_tile": f64["tile"]},
        "fp32_form": {"ratio_vs_fp64": value / value64, "errors_vs_fp64": errors,
                      "k_diffuse_fs_gbs": st32, "k_diffuse_fs_frac": st32 / peak,
                      "kernel_ms_per_step": per_step(f32["kernels"]), "stencil_tile": f32["tile"]},
        "roofline": roof,
        "e2e": e2e,
        "gpu_launches": f32["launches"],
        "clocks": f32["clocks"],
        "clocks_fp64": f64["clocks"],
        "cpu_baseline": cpu,
        "grain_check_vs_reference": check,
        "cfg2": cfg2,
    }
    print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def am_config(nsb, grains) -> dict:
    """config of both arms' lines (the same keys and values for the same run)."""
    return {"workload": "AM single-track melt pool, 512x256x128 cells, columnar substrate, FP32 form",
            "cells": AM_DIMS[0] * AM_DIMS[1] * AM_DIMS[2], "dx_m": AM_DX, "dt_s": AM_DT,
            "laser": {"speed_m_per_s": 0.5, "power_w": 150, "absorptivity": 0.4, "k_th": 100, "alpha": 3e-5},
            "substrate": {"top_plane": AM_TOP, "mean_width_m": AM_SUB_WIDTH, "seed": AM_SUB_SEED},
            "nsubblocks": list(nsb), "grains_after_run": grains,
            "l2": "inputs larger than L2 (fields about 0.7 GB FP32, 1.1 GB FP64)"}


def ds256_device(args, ws, stream, barrier, max_over_ranks) -> dict:
    """The 256^3 directional-solidification deck, device-timed K steps of each
    form (the cfg2 key of the default line)."""
    import torch
    import mumatscale_b200 as M
    K, Wm = args.steps, args.warmup
    td = tempfile.mkdtemp()
    deck = Path(td) / "ds.in"
    deck.write_text(deck_text())
    params = M.read_deck(deck)
    out = {}
    for form, prec in (("f64", M.PREC_F64), ("f32", M.PREC_F32)):
        with M.Domain(params, precision=prec) as dom:
            dom.set_stream(stream.cuda_stream)
            dom.autotune(reps=3)
            dom.step(Wm)
            torch.cuda.synchronize()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            dom.step(K)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1))
            dom.set_profiling(True)
            dom.step(K)
            torch.cuda.synchronize()
            ks = dom.kernel_stats()
            dom.set_profiling(False)
            kms, kn = ks["k_diffuse_fs"]
            gbs = BYTES_DIFFUSE[form] * N_CELL ** 3 / (kms / 1e3 / max(kn, 1)) / 1e9
            out[form] = {"value": ws * N_CELL ** 3 * K / (ms / 1e3), "ms_per_step": ms / K,
                         "k_diffuse_fs_gbs": gbs, "k_diffuse_fs_frac": gbs / measured_peak_gbs()[0]}
    out["workload"] = "multi-grain directional solidification, 256^3 cells"
    out["fp32_ratio_vs_fp64"] = out["f32"]["value"] / out["f64"]["value"]
    return out


def profile_arm(args) -> None:
    """Workload for ncu captures: one form, W + K steps, no timing, no CPU
    baseline.  --workload ds256 (default): the headline deck with --cells
    per edge; --workload am: the AM melt-pool deck scaled by --cells/256
    (x: 2 --cells, y: --cells, z: --cells/2) with its substrate.  Usage:
        ncu ... python bench.py --profile f64 --warmup 3 --steps 2"""
    import mumatscale_b200 as M
    td = tempfile.mkdtemp()
    deck = Path(td) / "bench.in"
    prec = M.PREC_F32 if args.profile == "f32" else M.PREC_F64
    if args.workload == "am":
        from mumatscale_b200 import workloads as W
        dims = (2 * args.cells, args.cells, args.cells // 2)
        deck.write_text(W.am_track(dims, 1e-6))
        dom = M.Domain(M.read_deck(deck), precision=prec)
        W.setup_substrate(dom, dims[2] - 8, 1e-6)
        ncell = dims[0] * dims[1] * dims[2]
    else:
        deck.write_text(deck_text(n=args.cells))
        dom = M.Domain(M.read_deck(deck), precision=prec)
        ncell = args.cells ** 3
    if args.tile != "auto":
        cpt, zc = (int(v) for v in args.tile.split(","))
        dom.set_stencil_tile(cpt, zc)
    if args.am_tile:
        dom.set_am_tile(args.am_tile)
    dom.step(args.warmup + args.steps)
    # --reduce R: R rounds of a step with the fraction-solid tile sums
    # (mms_step_reduce), a plain step and a field pass (mms_reduce)
    fs = []
    for _ in range(args.reduce):
        summed = dom.step_reduce(1, "fs_fraction")
        dom.step(1)
        fs.append((summed, dom.reduce("fs_fraction")))
    print(json.dumps({"profile": args.profile, "workload": args.workload, "cells": ncell,
                      "steps": args.warmup + args.steps + 2 * args.reduce, "grains": dom.num_grains,
                      "tma": dom.uses_tma, "tile": dom.stencil_tile(), "fs_fraction": fs}))
    dom.close()


def adjoint_workload(args) -> None:
    """Adjoint calibration: the one-grain deck at 128^3, 2000 steps recorded
    with checkpoints every 100; target ce from the same deck with D_l x 1.2
    and k x 0.9; gradient of 1/2 |ce - target|^2 w.r.t. (D_l, k, Gibbs-
    Thomson) by the FP64 and the FP32 adjoint, and central differences
    (step 1e-4 relative) of the FP64 frozen replay.  Prints one JSON line."""
    import torch
    import mumatscale_b200 as M
    from mumatscale_b200 import workloads as W
    n, steps, every, h = args.cells if args.cells != N_CELL else 128, 2000, 100, 1e-4
    deck, cells, thr, rot = W.one_grain(n)
    td = tempfile.mkdtemp()
    f = Path(td) / "adj.in"
    f.write_text(deck)
    p = M.read_deck(f)
    pt = M.read_deck(f)
    pt.Dliq *= 1.2
    pt.part_coef *= 0.9
    with M.Domain(pt) as d:
        W.setup_one_grain(d, cells, thr, rot)
        d.step(steps)
        target = d.download("ce")
    base = {"Dliq": p.Dliq, "part_coef": p.part_coef, "gibbs": p.gibbs_coef}
    out = {}
    for form, prec in (("f64", M.PREC_F64), ("f32", M.PREC_F32)):
        with M.Domain(p, precision=prec) as dom:
            W.setup_one_grain(dom, cells, thr, rot)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            dom.adjoint_record(steps, every)
            t1 = time.perf_counter()
            g = dom.adjoint_gradient(target)
            t2 = time.perf_counter()
            rec = {"loss": g["loss"], "dlogtheta": {k: g[k] * base[k] for k in base},
                   "forward_record_s": t1 - t0, "gradient_s": t2 - t1,
                   "grains": dom.num_grains, "fs_fraction": dom.reduce("fs_fraction")}
            if form == "f64":
                fd = {}
                t3 = time.perf_counter()
                for i, k in enumerate(base):
                    up, dn = [1.0] * 3, [1.0] * 3
                    up[i] += h
                    dn[i] -= h
                    fd[k] = (dom.adjoint_replay_loss(target, up) - dom.adjoint_replay_loss(target, dn)) / (2 * h)
                rec["fd"] = fd
                rec["fd_s"] = time.perf_counter() - t3
            out[form] = rec
    f64, f32 = out["f64"], out["f32"]
    big = max(abs(v) for v in f64["dlogtheta"].values())
    rel = {k: abs(f64["dlogtheta"][k] - f64["fd"][k]) / max(abs(f64["fd"][k]), 1e-6 * big) for k in base}
    rel32 = {k: abs(f32["dlogtheta"][k] - f64["dlogtheta"][k]) / max(abs(f64["dlogtheta"][k]), 1e-6 * big)
             for k in base}
    cells_n = n ** 3
    line = {"workload": f"adjoint calibration, one grain, {n}^3 cells, {steps} steps, checkpoints every {every}",
            "metric": "dL/dlog(theta) agreement; adjoint cell-updates/s", "data": "synthetic",
            "fp64": f64, "fp32": f32, "adjoint_vs_fd_rel": rel, "fp32_vs_fp64_rel": rel32,
            "fd_step_rel": h,
            "gradient_cell_updates_per_s": {"f64": cells_n * steps / f64["gradient_s"],
                                            "f32": cells_n * steps / f32["gradient_s"]}}
    print(json.dumps(line))


def ensemble_workload(args) -> None:
    """64 independent domains (edges from {32,48,64,96,128} per axis, cooling
    10-1000 K/s, nucleation 1e11-1e14 m^-3, seeded) in the FP32 form, stepped
    as one batch (one graph per step, one persistent stencil launch, tile
    autotuned) for 3000 steps; beside it (N=1) the same domains stepped one
    after another with mms_step.  Under torchrun the domains are dealt to
    the ranks by size (largest first to the least-loaded rank): no collective
    on the data path, timing is the max over ranks.  Rank 0 prints one JSON
    line."""
    import torch
    import mumatscale_b200 as M
    from mumatscale_b200 import workloads as W
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    decks = W.ensemble(64)
    td = Path(tempfile.mkdtemp())
    ps_all = []
    for i, d in enumerate(decks):
        f = td / f"e{i}.in"
        f.write_text(d)
        ps_all.append(M.read_deck(f))
    from mumatscale_b200.distributed import shard_balanced
    sizes = [p.gsdimx * p.gsdimy * p.gsdimz for p in ps_all]
    ps = [ps_all[i] for i in shard_balanced(sizes, ws)[rank]]
    cells_all = sum(sizes)
    steps = 3000 if args.steps == 200 else args.steps

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    with M.Batch(ps, precision=M.PREC_F32, device=dev) as b:
        tune = b.autotune(reps=3)
        b.step(args.warmup)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.step(steps)
        torch.cuda.synchronize()
        sec = max_over_ranks(time.perf_counter() - t0)
        barrier()
        grains = sum(d.num_grains - 1 for d in b.domains)
        tile = b.stencil_tile()
        launches = b.kernel_launches
    seq = None
    if ws == 1:
        # the same domains one after another (each its own graph), fewer steps
        seq_steps = min(steps, 300)
        doms = [M.Domain(p, precision=M.PREC_F32) for p in ps]
        for d in doms:
            d.step(args.warmup)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for d in doms:
            d.step(seq_steps)
        torch.cuda.synchronize()
        seq = {"value": cells_all * seq_steps / (time.perf_counter() - t0), "steps": seq_steps}
        for d in doms:
            d.close()
    if rank == 0:
        line = {"workload": "ensemble of 64 independent domains, edges {32,48,64,96,128}, FP32 form",
                "metric": UNIT, "unit": UNIT, "value": cells_all * steps / sec, "n_gpus": ws, "steps": steps,
                "warmup": args.warmup, "cells_total": cells_all, "ms_per_step": sec * 1e3 / steps,
                "scaling": "strong", "data": "synthetic",
                "tile": {"cells_per_thread": tile[0], "zchunk": tile[1], "persistent_ctas": tile[2],
                         "tuned_stencil_ms": tune[2]},
                "grains_rank0": grains, "kernel_launches_per_step": launches / max(1, steps + args.warmup),
                "sequential_domains": seq,
                "timing": "host clock around synchronised runs of device-resident steps, max over ranks"}
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def slabs_workload(args) -> None:
    """One 256^3 domain (the headline deck with NSubblocks 1 x 1 x 8) split
    into N z-slabs, one per rank (torchrun), exchanging boundary planes and
    new-grain lists over NCCL twice per step (mumatscale_b200.slabs): strong
    scaling of one domain.  FP64 plain form; device-timed with CUDA events on
    the slab's stream, max over ranks.  With one process it also times the
    same domain as 2 and 4 slabs on the one device (in-process group, device
    copies for the exchanges) beside the unsplit domain: the cost of the
    exchange points themselves.  Rank 0 prints one JSON line."""
    import datetime
    import torch
    import mumatscale_b200 as M
    from mumatscale_b200.slabs import DistributedSlab
    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    td = tempfile.mkdtemp()
    deck = Path(td) / "slabs.in"
    deck.write_text(deck_text(nsb=(1, 1, 8)))
    params = M.read_deck(deck)
    cells = N_CELL ** 3
    K, W = args.steps, args.warmup

    def max_over_ranks(x: float) -> float:
        if ws == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    if ws > 1:
        s = DistributedSlab(params, precision=M.PREC_F64, device=dev)
        s.dom.autotune(reps=5)  # stencil tile for this slab's grid
        s.step(W)
        st = s.stream
        run = s.step
        launches0 = s.dom.kernel_launches
    else:
        s = M.Domain(params, precision=M.PREC_F64, device=dev)
        st = torch.cuda.current_stream()
        s.set_stream(st.cuda_stream)
        s.autotune(reps=5)
        s.step(W)
        run = s.step
        launches0 = s.kernel_launches
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        e0.record(st)
        run(K)
        e1.record(st)
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    launches = (s.dom.kernel_launches if ws > 1 else s.kernel_launches) - launches0
    grains = s.dom.num_grains if ws > 1 else s.num_grains
    s.close()
    group = None
    if ws == 1:
        group = {}
        for n in (2, 4):
            with M.SlabGroup(params, n, precision=M.PREC_F64, devices=(dev,)) as g:
                for d in g.slabs:
                    d.autotune(reps=3)
                g.step(W)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                g.step(min(K, 100))
                torch.cuda.synchronize()
                sec = time.perf_counter() - t0
                group[f"{n}_slabs_one_device"] = {"value": cells * min(K, 100) / sec,
                                                  "ms_per_step": sec * 1e3 / min(K, 100)}
    if rank == 0:
        line = {"workload": "one 256^3 domain (NSubblocks 1 x 1 x 8) split into z-slabs, one per GPU, FP64",
                "metric": UNIT, "unit": UNIT, "value": cells * K / (ms / 1e3), "n_gpus": ws, "steps": K,
                "warmup": W, "ms_per_step": ms / K, "scaling": "strong", "data": "synthetic", "dtype": "f64",
                "parallelism": f"z-slabs x{ws}, NCCL send/recv of boundary planes + all-gathers per step",
                "gpu_launches": launches, "grains": grains, "clocks": clk.summary(),
                "one_device_groups": group,
                "timing": "CUDA events on the slab's stream around K steps, max over ranks"}
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def reference_arm(args) -> None:
    """The reference's own CPU path on the default (AM) deck, or on the 256^3
    directional deck with --workload ds256; rank 0 only."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    wl = "ds256" if args.workload == "ds256" else "am"
    res, why = run_reference(wl, args.warmup, args.steps)
    if not res:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    if wl == "am":
        config, dtype = am_config(res["nsubblocks"], res["grains"]), "f64"
        config["workload"] = config["workload"].replace("FP32 form", "the reference (FP64)")
    else:
        config = {"workload": "multi-grain directional solidification, 256^3 cells, FP64 plain form",
                  "cells": N_CELL ** 3, "dx_m": DX, "dt_s": DT, "G_K_per_m": 1e4, "V_m_per_s": 1e-3,
                  "nsubblocks": list(res["nsubblocks"]), "grains_after_run": res["grains"]}
        dtype = "f64"
    line = {
        "impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["sec"] * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic",
        "config": config, "parallelism": f"{res['procs']} MPI ranks on host cores",
        "cpu_baseline": {"value": res["value"], "unit": UNIT, "cores": res["procs"], "kind": "reference",
                         "sample": f"{args.steps} timesteps after {args.warmup}, NSubblocks {res['nsubblocks']}, "
                                   f"{res['procs']} MPI ranks through the shared-memory MPI shim"},
        "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=200,
                    help="timed steps of the CPU baseline leg (default: 2 on the AM deck, 200 on ds256)")
    ap.add_argument("--no-cfg2", action="store_true", help="leave the 256^3 directional deck out of the line")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", choices=["f64", "f32"], default=None,
                    help="run the workload for an ncu capture only")
    ap.add_argument("--cells", type=int, default=N_CELL, help="edge of the cubic domain (profile mode)")
    ap.add_argument("--reduce", type=int, default=0,
                    help="profile mode: rounds of (step with tile sums, plain step, field reduction) after the steps")
    ap.add_argument("--tile", default="auto", help="profile mode: stencil tile 'cells_per_thread,zchunk'")
    ap.add_argument("--am-tile", type=int, default=0,
                    help="profile mode: rows per tile of the FP32 AM contraction (mms_set_am_tile; 0 = default)")
    ap.add_argument("--workload", default=None, choices=["am", "ds256", "adjoint", "ensemble", "slabs"],
                    help="am: the AM melt-pool deck, the headline line (default); ds256, adjoint, "
                         "ensemble, slabs: the 256^3 directional-solidification, adjoint calibration, "
                         "batched-ensemble and one-domain-over-N-GPUs workloads (each its own JSON line). "
                         "With --profile the default is ds256.")
    args = ap.parse_args()
    if args.workload is None:
        args.workload = "ds256" if args.profile else "am"
    if args.warmup < 3:
        args.warmup = 3
    if args.profile:
        profile_arm(args)
    elif args.workload == "adjoint" and args.impl != "reference":
        adjoint_workload(args)
    elif args.workload == "ds256" and args.impl != "reference":
        ds256_workload(args)
    elif args.workload == "ensemble" and args.impl != "reference":
        ensemble_workload(args)
    elif args.workload == "slabs" and args.impl != "reference":
        slabs_workload(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
