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
    names = re.findall(r"^\s*(?:const\s+)?(?:void|int|size_t|char|unsigned\s+\w+|long\s+long|float|double)"
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


def test_every_export_group_is_declared():
    names = declared_functions()
    for n in ("ktmInterpLength", "ktmInterpTraces", "ktmSegyOpen", "ktmLoadSegySurvey",
              "ktmReadVelModel", "ktmIBM32toIEEEDevice", "ktmReleaseMemory", "ktmMemoryStats",
              "ktmCheckDeviceWaits", "ktmSelfTestDeviceWait",
              "ktmMigratePackedNoAlloc", "ktmLeastSquaresMigrate"):
        assert n in names, n


def _fake_job(ktm_lib, **over):
    from ktm._lib import KtmJob
    j = KtmJob()
    ktm_lib.ktmJobInit(C.byref(j))
    j.config.traceNo, j.config.tracePts, j.config.traceSampleRate = 4, 100, 0.004
    j.imageX.imagePnts = j.imageY.imagePnts = 2
    j.imageZ.imagePnts, j.imageZ.imageStep = 10, 0.004
    for name in ("midX", "midY", "offX", "offY", "traces", "velocity", "image"):
        setattr(j, name, 4096)     # non-NULL placeholders: every case fails before a copy
    j.deviceMemory = 1
    for k, v in over.items():
        setattr(j, k, v)
    return j


@pytest.mark.parametrize("over", [
    dict(weightMethod=2, pick=0),              # the fold takes the linear pick
    dict(weightMethod=2, tracesPacked=1, traceScale=4096, traceStride=104),   # not prefolded
    dict(traceFormat=3, tracesPacked=1),       # IBM words are raw traces
    dict(traceFormat=3, traceScale=4096),
    dict(weightMethod=9),
    dict(packFormat=7),
    dict(mode=5),
])
def test_job_combinations_rejected_without_device(ktm_lib, over):
    from ktm._lib import KTM_ERR_ARG
    j = _fake_job(ktm_lib, **over)
    assert ktm_lib.ktmMigrate(C.byref(j)) == KTM_ERR_ARG, ktm_lib.ktmGetLastErrorMessage()


def test_prepare_limits_without_device(ktm_lib):
    from ktm._lib import KTM_ERR_ARG, KTM_ERR_LIMIT, KtmPrep
    p = KtmPrep()
    p.traceNo, p.tracePts, p.sampleRate = 4, 20000, 0.002
    p.in_, p.out, p.outScale = 4096, 4096, 4096
    p.rho = 3                                   # FFT of 32768 > 16384 points
    assert ktm_lib.ktmPrepareTraces(C.byref(p)) == KTM_ERR_LIMIT
    p.rho, p.tracePts, p.inFormat = 0, 100, 9   # not F32 or IBM-32
    assert ktm_lib.ktmPrepareTraces(C.byref(p)) == KTM_ERR_ARG
    p.inFormat, p.outPitch = 0, 50              # pitch < tracePts + 2
    assert ktm_lib.ktmPrepareTraces(C.byref(p)) == KTM_ERR_ARG


def test_interp_limits_without_device(ktm_lib):
    from ktm._lib import KTM_ERR_ARG, KtmInterp
    assert ktm_lib.ktmInterpLength(1001, 2) == 4001
    assert ktm_lib.ktmInterpLength(1, 5) == 1
    assert ktm_lib.ktmInterpLength(0, 5) == 0
    q = KtmInterp()
    q.traceNo, q.tracePts, q.levels, q.in_, q.out = 3, 10, 11, 4096, 4096
    assert ktm_lib.ktmInterpTraces(C.byref(q)) == KTM_ERR_ARG        # levels > 10
    q.levels, q.outStride = 2, 20                                    # < 37 samples
    assert ktm_lib.ktmInterpTraces(C.byref(q)) == KTM_ERR_ARG


def test_demigrate_pitch_rejected_without_device(ktm_lib):
    from ktm._lib import KTM_ERR_ARG
    j = _fake_job(ktm_lib)
    assert ktm_lib.ktmDemigrate(C.byref(j), C.c_void_p(4096), 101) == KTM_ERR_ARG  # < nt + 2


def test_header_compiles_as_c_and_cpp_and_links(tmp_path, ktm_lib):
    """A C caller of the reference's kind: include/ktm.h compiles as C11 and C++17,
    and a program using the drop-in's host helpers links against libktm.so and runs
    without a GPU."""
    import shutil
    import subprocess
    import ktm
    if shutil.which("gcc") is None or shutil.which("g++") is None:
        pytest.skip("no host compiler")
    inc = os.path.join(ROOT, "include")
    src = tmp_path / "caller.c"
    src.write_text(
        '#include <stdio.h>\n#include "ktm.h"\n'
        "int main(void) {\n"
        "  struct imageGrid gx = {3, 12.5f, 100.0f}, gy = {2, 25.0f, 0.0f}, gz = {4, 0.002f, 0.0f};\n"
        "  float xx[3], yy[2], zz[4];\n"
        "  initThreeAxes(&gx, &gy, &gz, xx, yy, zz);\n"
        '  printf("%.4f %.4f %.4f %s\\n", xx[2], yy[1], zz[3], ktmGetErrorString(KTM_ERR_LIMIT));\n'
        "  return 0;\n}\n")
    for cc, std, name in (("gcc", "-std=c11", "c"), ("g++", "-std=c++17", "cpp")):
        r = subprocess.run([cc, std, "-Wall", "-Werror", "-fsyntax-only", "-x",
                            "c" if name == "c" else "c++", "-I" + inc, str(src)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    libdir = os.path.dirname(ktm.LIB_PATH)
    exe = tmp_path / "caller"
    r = subprocess.run(["gcc", "-std=c11", "-I" + inc, str(src), "-o", str(exe), "-L" + libdir, "-lktm",
                        "-Wl,-rpath," + libdir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    x, y, z, msg = r.stdout.split(" ", 3)
    assert (float(x), float(y), float(z)) == (125.0, 25.0, 0.006) and msg.strip()


def test_memory_stats_counter_without_device(ktm_lib):
    """The allocation counter is host state: readable without a GPU (and no call
    on the CPU has allocated)."""
    n = C.c_ulonglong(123)
    assert ktm_lib.ktmMemoryStats(C.byref(n), None, None) == 0
    assert n.value == 0
