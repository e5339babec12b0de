"""The bounded device-side waits end with an error status, not a hang.

The interface-list kernel's decoupled look-back (each list block waits for
the status words of the blocks before it) is the wait made to run out: the
test hook holds back one block's status word, a flag that nothing else
writes, and shortens the poll bound.  No device fault is caused: the wait
gives up, the kernel raises MMS_ERR_TIMEOUT in the control block, later
kernels of the step do nothing, and the call returns the status.  The
device stays usable: a fresh context on it reproduces the reference's
golden state."""
from __future__ import annotations

import pytest

import mumatscale_b200 as M
from conftest import golden, golden_deck
from digests import mismatches, state_digests

MMS_ERR_TIMEOUT = 9


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [M.PREC_F64, M.PREC_F32])
def test_lookback_wait_runs_out(built, cuda_device, prec):
    p = M.read_deck(golden_deck("small4"))
    dom = M.Domain(p, precision=prec)
    dom.step(5)
    dom.test_hold_list_block(0, polls=2000)
    with pytest.raises(M.MmsError) as e:
        dom.step(1)
    assert e.value.status == MMS_ERR_TIMEOUT
    dom.close()
    # the device is usable: a new context reaches the reference's state
    rec = golden("small4")
    with M.Domain(p, precision=M.PREC_F64) as fresh:
        fresh.step(50)
        assert mismatches(state_digests(fresh), rec["steps"]["50"]["digest"]) == []


def test_hold_hook_arguments(built):
    """Argument checks happen on the host (no device needed)."""
    lib = M.load_library()
    assert lib.mms_test_hold_list_block(None, 0, 0) == 1  # MMS_ERR_ARG
