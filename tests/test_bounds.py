"""The bounds-checked build, libmms_b200_bounds.so (kernels compiled with
-DMMS_BOUNDS): every checked kernel index outside its buffer raises
MMS_ERR_BOUNDS and skips the access, so an overrun shows up as a failing
call instead of a memory fault.  The reference has no sanitizer; its GPU
build builds lists with atomic captures (growth.c:507, grain.c:1274).

CPU: the library builds and exports what include/mms.h declares.  GPU: the
bit-exact parity tests (golden decks, slabs, reductions, batches) run again
against it in a child process (MMS_LIBRARY selects the library) and must
pass unchanged: no index leaves its buffer and the checks change no result."""
from __future__ import annotations

import os
import re
import subprocess
import sys

import pytest

from conftest import ROOT
from test_host import declared_functions


def _bounds_library():
    from mumatscale_b200 import build as b
    return b.build(bounds=True)


def test_bounds_library_exports_every_declared_symbol(built):
    lib = _bounds_library()
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (mms_\w+)", out))
    assert set(declared_functions()) <= exported


@pytest.mark.gpu
def test_parity_suite_under_bounds_checks(built, cuda_device):
    lib = _bounds_library()
    env = dict(os.environ, MMS_LIBRARY=str(lib))
    probe = subprocess.run([sys.executable, "-c", "import mumatscale_b200 as M; print(M.load_library()._name)"],
                           cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert probe.returncode == 0 and probe.stdout.strip() == str(lib), probe.stdout + probe.stderr
    tests = ["tests/test_gpu_parity.py::test_fp64_bit_exact_vs_reference",
             "tests/test_gpu_parity.py::test_fp64_matches_oracle_every_step",
             "tests/test_slabs.py", "tests/test_reductions.py", "tests/test_batch.py"]
    r = subprocess.run([sys.executable, "-m", "pytest", "-x", "-q", "-m", "gpu", "-p", "no:cacheprovider", *tests],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert " passed" in r.stdout
