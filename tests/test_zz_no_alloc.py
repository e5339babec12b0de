"""mms_reduce_field_noalloc through the C ABI: the same sums as mms_reduce,
taken over caller-owned device fields with library-owned fixed scratch.

The file name sorts last so the GPU test also runs after every other test
has used the device."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import mumatscale_b200 as M
from conftest import golden_deck

MMS_ERR_ARG = 1
MMS_ERR_NO_DEVICE = 3
MMS_ERR_SCRATCH_LIMIT = 12
REDUCE = {"fs_fraction": 0, "solid_volume": 1, "ce_sum": 2}
# Both sums are FP64 with compensation; only the summation order differs.
REL_TOL = 1e-13


def _noalloc():
    fn = M.load_library().mms_reduce_field_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                   C.c_void_p, C.c_void_p]
    return fn


def test_noalloc_rejects_before_device_work(built):
    """Argument and size checks come before any CUDA call: on a machine
    without a GPU an oversized grid still reports the scratch limit."""
    fn = _noalloc()
    dummy = C.c_void_p(16)  # never dereferenced: every call below is rejected on the host
    assert fn(dummy, 0, 1025, 1024, 1024, 0, 1e-6, dummy, None) == MMS_ERR_SCRATCH_LIMIT
    assert fn(dummy, 0, 0, 8, 8, 0, 1e-6, dummy, None) == MMS_ERR_ARG
    assert fn(dummy, 2, 8, 8, 8, 0, 1e-6, dummy, None) == MMS_ERR_ARG
    assert fn(dummy, 0, 8, 8, 8, 3, 1e-6, dummy, None) == MMS_ERR_ARG
    assert fn(None, 0, 8, 8, 8, 0, 1e-6, dummy, None) == MMS_ERR_ARG
    assert b"scratch" in M.load_library().mms_status_string(MMS_ERR_SCRATCH_LIMIT)


def _stepped_small4():
    """small4 after 300 steps: a few thousand cells, one partial-sum block."""
    p = M.read_deck(golden_deck("small4"))
    with M.Domain(p, precision=M.PREC_F64) as dom:
        dom.step(300)
        fields = {"fs": dom.download("fs"), "ce": dom.download("ce")}
        want = {w: dom.reduce(w) for w in REDUCE}
    return p, fields, want


def _ragged_uploaded():
    """A 70 x 50 x 40 grid (140,000 interior cells: eight full partial-sum
    blocks and a ninth partial one) holding seeded fields with fs partly above
    1, so the clamp of the fraction-solid sums matters, uploaded into a
    context whose own reductions give the expected values."""
    from mumatscale_b200 import workloads as W
    import tempfile
    from pathlib import Path
    deck, _, _, _ = W.one_grain(8)
    text = deck.replace("NCellsPerSB 8 8 8", "NCellsPerSB 70 50 40")
    assert text != deck
    f = Path(tempfile.mkdtemp()) / "ragged.in"
    f.write_text(text)
    p = M.read_deck(f)
    rng = np.random.default_rng(7)
    shape = (42, 52, 72)
    fs = rng.uniform(-0.05, 1.2, shape)
    ce = rng.uniform(3.0, 6.0, shape)
    with M.Domain(p, precision=M.PREC_F64) as dom:
        dom.upload("fs", fs)
        dom.upload("ce", ce)
        fields = {"fs": dom.download("fs"), "ce": dom.download("ce")}
        want = {w: dom.reduce(w) for w in REDUCE}
    assert fields["fs"].shape == shape
    return p, fields, want


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["small4", "ragged_multiblock"])
def test_noalloc_matches_mms_reduce(built, cuda_device, case):
    import torch
    fn = _noalloc()
    p, fields, want = _stepped_small4() if case == "small4" else _ragged_uploaded()
    gz, gy, gx = (s - 2 for s in fields["fs"].shape)
    assert 0 < want["fs_fraction"] < 1
    nblocks = -(-gx * gy * gz // 16384)
    assert (nblocks == 1) == (case == "small4")

    dev = torch.device("cuda", cuda_device)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    d64 = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in fields.items()}
    d32 = {k: v.to(torch.float32) for k, v in d64.items()}
    out = torch.empty(1, dtype=torch.float64, device=dev)

    def run(field: torch.Tensor, dtype: int, what: str) -> float:
        out.fill_(float("nan"))
        st = fn(field.data_ptr(), dtype, gx, gy, gz, REDUCE[what], p.cellSize, out.data_ptr(),
                stream.cuda_stream)
        assert st == 0, M.load_library().mms_status_string(st)
        stream.synchronize()
        return float(out.item())

    for call in range(2):  # the scratch is reused: two calls in a row agree
        for what in REDUCE:
            src = "ce" if what == "ce_sum" else "fs"
            got = run(d64[src], M.PREC_F64, what)
            assert abs(got - want[what]) <= REL_TOL * abs(want[what]), (call, what, got, want[what])
            # FP32 input: the same sum over the rounded values
            x = fields[src][1:-1, 1:-1, 1:-1].astype(np.float32).astype(np.float64)
            if what != "ce_sum":
                x = np.minimum(x, 1.0)
            ref = float(np.sum(x, dtype=np.float64))
            if what == "solid_volume":
                ref *= p.cellSize ** 3
            elif what == "fs_fraction":
                ref = ref * p.cellSize ** 3 / (gx * gy * gz * p.cellSize ** 3)
            got32 = run(d32[src], M.PREC_F32, what)
            assert abs(got32 - ref) <= 1e-12 * abs(ref), (call, what, got32, ref)
