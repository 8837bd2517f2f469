"""libktm.so on the CPU: it loads, exports every entry point include/ktm.h
declares, lays out ktm_job as the bindings do, and rejects bad arguments
before touching the device."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ktm.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:void|int|size_t|char|unsigned\s+\w+|float|double)"
                       r"\s*\**\s*(\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_dropins():
    names = declared_functions()
    for n in ("ktmMigrationCPU", "ktmMigrationGPU", "initThreeAxes", "initTwoAxes", "ktmMigrate"):
        assert n in names


def test_library_exports_every_declared_function(ktm_lib):
    missing = [n for n in declared_functions() if not hasattr(ktm_lib, n)]
    assert not missing, missing


def test_job_struct_layout(ktm_lib):
    from ktm._lib import KtmJob
    assert ktm_lib.ktmJobStructSize() == C.sizeof(KtmJob)


def test_null_job_rejected_without_device(ktm_lib):
    from ktm._lib import KTM_ERR_ARG
    assert ktm_lib.ktmMigrate(None) == KTM_ERR_ARG
    assert ktm_lib.ktmGetLastError() == KTM_ERR_ARG
    assert b"NULL" in ktm_lib.ktmGetLastErrorMessage()


def test_bad_enums_rejected_without_device(ktm_lib):
    from ktm._lib import KTM_ERR_ARG, KtmJob
    j = KtmJob()
    ktm_lib.ktmJobInit(C.byref(j))
    j.traceFormat = 7
    assert ktm_lib.ktmMigrate(C.byref(j)) == KTM_ERR_ARG
    ktm_lib.ktmJobInit(C.byref(j))
    j.pick = 5
    assert ktm_lib.ktmMigrate(C.byref(j)) == KTM_ERR_ARG
    ktm_lib.ktmJobInit(C.byref(j))
    j.config.traceNo, j.config.tracePts, j.config.traceSampleRate = 4, 10, 0.0
    j.imageZ.imagePnts = 0
    for name in ("midX", "midY", "offX", "offY", "traces"):
        setattr(j, name, 8)   # non-NULL placeholders: rejected before any copy
    assert ktm_lib.ktmMigrate(C.byref(j)) == KTM_ERR_ARG    # sample rate 0


def test_dropin_null_grid_records_error(ktm_lib):
    from ktm._lib import KTM_ERR_ARG
    ktm_lib.ktmMigrationCPU(None, None, None, None, None, None, None, None, None, None, None)
    assert ktm_lib.ktmGetLastError() == KTM_ERR_ARG


def test_init_three_axes_matches_reference_arithmetic(ktm_lib):
    import numpy as np
    import ktm
    import oracle
    gx, gy, gz = ktm.grid(17, 12.5, -3.25), ktm.grid(3, 0.1, 0.7), ktm.grid(1001, 0.002, 0.0)
    xx, yy, zz = ktm.initThreeAxes(gx, gy, gz)
    for g, a in ((gx, xx), (gy, yy), (gz, zz)):
        i = np.arange(g.imagePnts, dtype=np.float32)
        expect = (np.float32(g.imageStart) + (i * np.float32(g.imageStep)).astype(np.float32))
        assert np.array_equal(a.view(np.uint32), expect.astype(np.float32).view(np.uint32))
    assert oracle is not None


def test_error_strings(ktm_lib):
    for code in range(8):
        assert ktm_lib.ktmGetErrorString(code)
