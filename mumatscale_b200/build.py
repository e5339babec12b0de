"""Builds the in-tree native artifacts of mumatscale_b200.

    libmms_b200.so         the C-ABI library (include/mms.h): sm_100a kernels
                           and the host side, CUDA runtime linked statically
    libmms_b200_bounds.so  the same with kernel index checks (-DMMS_BOUNDS):
                           an index outside its buffer raises MMS_ERR_BOUNDS
                           and the access is skipped; selected at run time by
                           MMS_LIBRARY=<path> (tests/test_bounds.py)
    mmsb200                the command-line driver (ca_main.c interface)

Everything is compiled for sm_100a only.  Device code is compiled with
-fmad=false so FP64 results match the reference's x86-64 build bit for bit.
Usage:  python -m mumatscale_b200.build  [--force] [--bounds]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libmms_b200.so"
BUILD_BOUNDS = PKG / "_build_bounds"
LIB_BOUNDS = PKG / "libmms_b200_bounds.so"
EXE = PKG / "mmsb200"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++"
CC = "/usr/bin/gcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["kernels.cu", "mms_api.cu", "adjoint.cu", "am_tc.cu", "noalloc.cu", "sites.cu"]
CXX_SOURCES = ["deck.cpp", "host_setup.cpp", "output.cpp"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ({r.returncode})")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, bounds: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "mms.h"]
    if bounds:
        build(force, verbose)  # the host objects are shared
        BUILD_BOUNDS.mkdir(exist_ok=True)
    objs = []
    for src in CU_SOURCES:
        obj = (BUILD_BOUNDS if bounds else BUILD) / (src + ".o")
        if force or _stale(obj, [CSRC / src] + headers):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
                   "-Xcompiler", "-fPIC", "-Xptxas", "-v" if verbose else "-O3",
                   *(["-DMMS_BOUNDS"] if bounds else []),
                   "-c", str(CSRC / src), "-o", str(obj)]
            _run(cmd)
        objs.append(obj)
    if bounds:
        objs += [BUILD / (src + ".o") for src in CXX_SOURCES]
        if force or _stale(LIB_BOUNDS, objs):
            _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB_BOUNDS), *map(str, objs),
                  "-Xlinker", "--no-undefined", "-lz", "-lpthread", "-ldl", "-lrt"])
        return LIB_BOUNDS
    for src in CXX_SOURCES:
        obj = BUILD / (src + ".o")
        if force or _stale(obj, [CSRC / src] + headers):
            _run([CXX, "-O2", "-fPIC", "-std=c++17", "-Wall", "-c", str(CSRC / src), "-o", str(obj)])
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs),
              "-Xlinker", "--no-undefined", "-lz", "-lpthread", "-ldl", "-lrt"])
    main_src = CSRC / "mms_main.c"
    if force or _stale(EXE, [main_src, LIB, ROOT / "include" / "mms.h"]):
        _run([CC, "-O2", "-std=gnu11", "-o", str(EXE), str(main_src), str(LIB),
              "-Wl,-rpath,$ORIGIN"])
    return LIB


def build_oracle(reference_present: bool | None = None) -> None:
    """Builds the CPU checkers under oracle/_ref (test infrastructure)."""
    oracle = ROOT / "oracle"
    _run(["make", "-C", str(oracle), "oracle"])
    # the reference's sources: REF_SRC, the same variable oracle/Makefile reads
    ref_src = os.environ.get("REF_SRC", "/root/reference/src")
    if reference_present is None:
        reference_present = Path(ref_src).is_dir()
    if reference_present:
        _run(["make", "-C", str(oracle), "ref", f"REF_SRC={ref_src}"])


if __name__ == "__main__":
    force = "--force" in sys.argv
    if force and BUILD.exists():
        shutil.rmtree(BUILD)
    print(build(force=force, verbose="-v" in sys.argv, bounds="--bounds" in sys.argv))
