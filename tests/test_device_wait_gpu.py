"""Bounded device waits of the fast kernels (needs a B200).

The fast kernels stage each chunk of packed trace rows into shared memory with
one bulk (TMA) copy completed on an mbarrier, and every wait on it is bounded.
The failure is made without a GPU fault: the self-test waits on a barrier that
nothing arrives on, so the bound runs out, the wait is counted on the device,
the host reads KTM_ERR_TIMEOUT, and the context stays usable for the next
migration.
"""
from __future__ import annotations

import pytest

import oracle
from test_parity_gpu import fast, random_case, rel_l2

pytestmark = pytest.mark.gpu

KTM_OK, KTM_ERR_ARG, KTM_ERR_TIMEOUT = 0, 1, 6


def test_bulk_copy_lands_and_wait_bound_reports(cuda, ktm_lib):
    assert ktm_lib.ktmCheckDeviceWaits() == KTM_OK          # nothing counted so far
    assert ktm_lib.ktmSelfTestDeviceWait(0, 100) == KTM_OK   # copy lands, bytes checked
    assert ktm_lib.ktmSelfTestDeviceWait(1, 20) == KTM_ERR_TIMEOUT
    assert b"ran out" in ktm_lib.ktmGetLastErrorMessage()
    assert ktm_lib.ktmCheckDeviceWaits() == KTM_OK          # the count was reset
    assert ktm_lib.ktmSelfTestDeviceWait(0, 0) == KTM_ERR_ARG

    # the context is still usable: a fast migration after the timed-out wait
    case = random_case(23, ntr=211, nx=7, ny=3, nz=150, data="ricker")
    img = fast(cuda, case, pick="linear")
    assert ktm_lib.ktmCheckDeviceWaits() == KTM_OK
    assert rel_l2(img, oracle.migrate_f64(*case, pick=1, prefold=0)) < 1e-3
