"""The bounded waits of the grid exchange, made to run out on the device.

Every PCG kernel's grid exchange waits for the other blocks of its group through an
arrival counter; each wait gives up after a bounded number of polls, records a timeout
and lets the kernel finish normally (no trap, no hang), and the host reports
PK_ERR_TIMEOUT / PK_FLAG_BARRIER_TIMEOUT.  pk_exchange_wait_selftest runs that exchange
code in one cooperative launch whose group names more members than were launched, so the
counter target cannot be reached: every block must give up and report it, and the GPU
context must stay usable for the next launch and the next step.
"""
import ctypes as C

import numpy as np
import pytest

from physik_b200 import meshes

pytestmark = pytest.mark.gpu

L = pytest.importorskip("physik_b200._lib")
from physik_b200.world import SimWorld  # noqa: E402

PK_ERR_TIMEOUT = -6


def selftest(blocks, missing, limit):
    out = np.full((blocks, 3), -1.0)
    rc = L.PK.pk_exchange_wait_selftest(0, blocks, missing, limit, out.ctypes.data_as(C.c_void_p))
    return rc, out


@pytest.mark.parametrize("blocks", [2, 37, 64])
def test_complete_group_exchanges(blocks):
    rc, out = selftest(blocks, 0, 1 << 22)
    assert rc == 0
    assert np.all(out[:, 0] == 1.0)
    assert np.all(out[:, 1] == blocks * (blocks + 1) / 2) and np.all(out[:, 2] == blocks)


@pytest.mark.parametrize("missing", [1, 5])
def test_missing_member_times_out_and_the_context_stays_usable(missing):
    rc, out = selftest(16, missing, 1 << 12)
    assert rc == PK_ERR_TIMEOUT
    assert np.all(out[:, 0] == 0.0)  # every block gave up and left through its normal exit
    # the same exchange with every member present still completes afterwards
    rc, out = selftest(16, 0, 1 << 22)
    assert rc == 0 and np.all(out[:, 0] == 1.0)
    # and a step on the same device runs clean
    w = SimWorld(meshes.small_box(3, 2, 2), precision="mixed")
    w.step()
    st = w.cg_stats()
    assert st["flags"] & L.FLAG_INTEGRATED and not (st["flags"] & L.FLAG_BARRIER_TIMEOUT)


def test_bad_arguments_are_refused_without_a_launch():
    out = np.zeros((4, 3))
    p = out.ctypes.data_as(C.c_void_p)
    assert L.PK.pk_exchange_wait_selftest(0, 1, 0, 100, p) == -3
    assert L.PK.pk_exchange_wait_selftest(0, 4, 0, 0, p) == -3
    assert L.PK.pk_exchange_wait_selftest(0, 4, 0, 100, None) == -3
