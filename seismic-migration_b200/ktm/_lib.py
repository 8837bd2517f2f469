"""ctypes binding of libktm.so (the C ABI declared in include/ktm.h).

The library is built in-tree by ``seismic-migration_b200/build.py``.  There is
no fallback: if ``libktm.so`` is missing or cannot be loaded, every call fails
with ``KtmError``.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libktm.so")

# status codes (ktm.h)
KTM_OK = 0
KTM_ERR_ARG = 1
KTM_ERR_CUDA = 2
KTM_ERR_NOMEM = 3
KTM_ERR_LIMIT = 4
KTM_ERR_IO = 5
KTM_ERR_TIMEOUT = 6
KTM_ERR_NODEVICE = 7

KTM_MODE_REFERENCE, KTM_MODE_FAST, KTM_MODE_F64 = 0, 1, 2
KTM_FMT_F32, KTM_FMT_F16, KTM_FMT_BF16, KTM_FMT_IBM32, KTM_FMT_F64 = 0, 1, 2, 3, 4
KTM_PICK_TRUNCATE, KTM_PICK_LINEAR = 0, 1
KTM_RHO_NONE, KTM_RHO_2D, KTM_RHO_25D, KTM_RHO_3D = 0, 1, 2, 3


class KtmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ktm error {code}: {msg}")
        self.code = code


class ImageGrid(C.Structure):
    """struct imageGrid (psktmFunctions.c:10-14 field names)."""
    _fields_ = [("imagePnts", C.c_int), ("imageStep", C.c_float), ("imageStart", C.c_float)]

    def axis(self):
        import numpy as np
        i = np.arange(self.imagePnts, dtype=np.float32)
        return (np.float32(self.imageStart) + i * np.float32(self.imageStep)).astype(np.float32)


class JobParams(C.Structure):
    """struct jobParams (psktmCPU.c:29,59,82 field names)."""
    _fields_ = [("traceNo", C.c_int), ("tracePts", C.c_int), ("traceSampleRate", C.c_float)]


P = C.c_void_p


class KtmJob(C.Structure):
    """ktm_job (include/ktm.h)."""
    _fields_ = [
        ("imageX", ImageGrid), ("imageY", ImageGrid), ("imageZ", ImageGrid),
        ("config", JobParams),
        ("midX", P), ("midY", P), ("offX", P), ("offY", P),
        ("traces", P), ("traceScale", P),
        ("traceFormat", C.c_int), ("traceStride", C.c_int), ("tracesPacked", C.c_int),
        ("tracesPrefolded", C.c_int),
        ("velocity", P), ("velocityCube", C.c_int),
        ("image", P),
        ("mode", C.c_int), ("pick", C.c_int), ("aperture", C.c_float),
        ("accumulate", C.c_int), ("deviceMemory", C.c_int),
        ("stream", P),
        ("tileRun", C.c_int), ("tileCols", C.c_int),
        ("pairsEvaluated", P),
        ("rho", C.c_int), ("packFormat", C.c_int), ("weightMethod", C.c_int),
        ("tileChunk", C.c_int),
    ]


class KtmTile(C.Structure):
    """ktm_tile (include/ktm.h)."""
    _fields_ = [("tileRun", C.c_int), ("tileCols", C.c_int), ("tileChunk", C.c_int),
                ("ctasPerSm", C.c_int), ("ms", C.c_float)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class KtmPrep(C.Structure):
    """ktm_prep (include/ktm.h)."""
    _fields_ = [
        ("traceNo", C.c_int), ("tracePts", C.c_int), ("inStride", C.c_int),
        ("sampleRate", C.c_float), ("in_", P), ("rho", C.c_int), ("rhoScriptOrder", C.c_int),
        ("prefold", C.c_int), ("outFormat", C.c_int), ("outPitch", C.c_int), ("out", P),
        ("outScale", P), ("stream", P), ("inFormat", C.c_int),
    ]


class KtmLsm(C.Structure):
    """ktm_lsm (include/ktm.h)."""
    _fields_ = [
        ("job", KtmJob), ("data", P), ("dataPitch", C.c_int), ("model", P),
        ("iterations", C.c_int), ("useGraph", C.c_int), ("residualNorms", P),
        ("gradientNorms", P),
    ]


class KtmInp(C.Structure):
    """ktm_inp (include/ktm.h): the 12 numbers of inp.txt."""
    _fields_ = [("tracePts", C.c_int), ("sampleRate", C.c_float), ("traceNo", C.c_int),
                ("x", ImageGrid), ("y", ImageGrid), ("z", ImageGrid)]


class KtmSurvey(C.Structure):
    """ktm_survey (include/ktm.h): one data directory read by ktmLoadSurvey."""
    _fields_ = [("inp", KtmInp), ("traces", P), ("traceFormat", C.c_int),
                ("midX", P), ("midY", P), ("offX", P), ("offY", P),
                ("velocity", P), ("velocityCube", C.c_int),
                ("originX", C.c_double), ("originY", C.c_double)]


class KtmSegyInfo(C.Structure):
    """ktm_segy_info (include/ktm.h)."""
    _fields_ = [("text", C.c_char * 3240), ("reel32", C.c_uint * 3), ("reel16", C.c_uint * 24),
                ("sampleInterval", C.c_int), ("samplesPerTrace", C.c_int), ("format", C.c_int),
                ("bigEndian", C.c_int), ("traceBytes", C.c_longlong), ("traceCount", C.c_longlong)]


class KtmSegyTrace(C.Structure):
    """ktm_segy_trace (include/ktm.h)."""
    _fields_ = [("values", C.c_int * 101), ("srcX", C.c_double), ("srcY", C.c_double),
                ("recX", C.c_double), ("recY", C.c_double)]


class KtmInterp(C.Structure):
    """ktm_interp (include/ktm.h)."""
    _fields_ = [("traceNo", C.c_int), ("tracePts", C.c_int), ("levels", C.c_int),
                ("in_", P), ("inStride", C.c_int), ("out", P), ("outStride", C.c_longlong),
                ("stream", P)]


_lib = None


def lib() -> C.CDLL:
    """Load libktm.so once; raise if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise KtmError(-1, f"{LIB_PATH} is not built: run seismic-migration_b200/build.py")
    L = C.CDLL(LIB_PATH)
    G = C.POINTER(ImageGrid)
    J = C.POINTER(JobParams)
    L.ktmMigrationCPU.argtypes = [G, G, G, J] + [P] * 7
    L.ktmMigrationCPU.restype = None
    L.ktmMigrationGPU.argtypes = [G, G, G, J] + [P] * 7
    L.ktmMigrationGPU.restype = None
    L.initThreeAxes.argtypes = [G, G, G, P, P, P]
    L.initThreeAxes.restype = None
    L.initTwoAxes.argtypes = [G, G, P, P]
    L.initTwoAxes.restype = None
    L.ktmGetLastError.restype = C.c_int
    L.ktmGetLastErrorMessage.restype = C.c_char_p
    L.ktmGetErrorString.argtypes = [C.c_int]
    L.ktmGetErrorString.restype = C.c_char_p
    L.ktmJobInit.argtypes = [C.POINTER(KtmJob)]
    L.ktmJobInit.restype = None
    L.ktmJobStructSize.restype = C.c_size_t
    L.ktmMigrate.argtypes = [C.POINTER(KtmJob)]
    L.ktmMigrate.restype = C.c_int
    L.ktmMigrateColumnsF64.argtypes = [C.POINTER(KtmJob), P, C.c_int, P]
    L.ktmMigrateColumnsF64.restype = C.c_int
    L.ktmPackedPitch.argtypes = [C.c_int, C.c_int]
    L.ktmPackedPitch.restype = C.c_int
    L.ktmPrepareTraces.argtypes = [C.POINTER(KtmPrep)]
    L.ktmPrepareTraces.restype = C.c_int
    L.ktmDemigrate.argtypes = [C.POINTER(KtmJob), P, C.c_int]
    L.ktmDemigrate.restype = C.c_int
    L.ktmVrmsGradient.argtypes = [C.POINTER(KtmJob), P]
    L.ktmVrmsGradient.restype = C.c_int
    L.ktmLeastSquaresMigrate.argtypes = [C.POINTER(KtmLsm)]
    L.ktmLeastSquaresMigrate.restype = C.c_int
    L.ktmMigrateBatch.argtypes = [C.POINTER(KtmJob), C.c_int, P]
    L.ktmMigrateBatch.restype = C.c_int
    L.ktmAutotune.argtypes = [C.POINTER(KtmJob), C.POINTER(C.c_int)]
    L.ktmAutotune.restype = C.c_int
    L.ktmAutotuneTile.argtypes = [C.POINTER(KtmJob), C.POINTER(KtmTile)]
    L.ktmAutotuneTile.restype = C.c_int
    L.ktmTileCandidates.argtypes = [C.POINTER(KtmJob), C.POINTER(KtmTile), C.c_int,
                                    C.POINTER(C.c_int)]
    L.ktmTileCandidates.restype = C.c_int
    L.ktmMigratePackedNoAlloc.argtypes = [C.POINTER(KtmJob)]
    L.ktmMigratePackedNoAlloc.restype = C.c_int
    L.ktmProbePeaks.argtypes = [P, P, P]
    L.ktmProbePeaks.restype = C.c_int
    L.ktmSynthesizeTraces.argtypes = [C.c_int, C.c_int, C.c_float, P, P, P, P, C.c_int, P,
                                      C.c_double, C.c_double, C.c_ulonglong, C.c_int, P, P]
    L.ktmSynthesizeTraces.restype = C.c_int
    L.ktmReadInp.argtypes = [C.c_char_p, C.POINTER(KtmInp)]
    L.ktmReadInp.restype = C.c_int
    L.ktmWriteInp.argtypes = [C.c_char_p, C.POINTER(KtmInp)]
    L.ktmWriteInp.restype = C.c_int
    L.ktmLoadSurvey.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(KtmSurvey)]
    L.ktmLoadSurvey.restype = C.c_int
    L.ktmFreeSurvey.argtypes = [C.POINTER(KtmSurvey)]
    L.ktmFreeSurvey.restype = None
    L.ktmWriteImage.argtypes = [C.c_char_p, P, C.c_size_t]
    L.ktmWriteImage.restype = C.c_int
    L.ktmIBM32toIEEE.argtypes = [P, P, C.c_int]
    L.ktmIBM32toIEEE.restype = None
    L.ktmIBM32toIEEEDevice.argtypes = [P, P, C.c_size_t, P]
    L.ktmIBM32toIEEEDevice.restype = C.c_int
    L.ktmSegyOpen.argtypes = [C.c_char_p, C.c_int, C.POINTER(KtmSegyInfo)]
    L.ktmSegyOpen.restype = C.c_int
    L.ktmSegyReadTraces.argtypes = [C.c_char_p, C.POINTER(KtmSegyInfo), C.c_longlong,
                                    C.c_longlong, P, C.POINTER(KtmSegyTrace)]
    L.ktmSegyReadTraces.restype = C.c_int
    L.ktmSegyTraceFormat.argtypes = [C.POINTER(KtmSegyInfo)]
    L.ktmSegyTraceFormat.restype = C.c_int
    L.ktmLoadSegySurvey.argtypes = [C.c_char_p, C.c_int, C.c_longlong, C.c_longlong, C.c_int,
                                    C.POINTER(KtmSurvey)]
    L.ktmLoadSegySurvey.restype = C.c_int
    L.ktmInterpLength.argtypes = [C.c_int, C.c_int]
    L.ktmInterpLength.restype = C.c_longlong
    L.ktmInterpTraces.argtypes = [C.POINTER(KtmInterp)]
    L.ktmInterpTraces.restype = C.c_int
    L.ktmReleaseMemory.argtypes = []
    L.ktmReleaseMemory.restype = C.c_int
    L.ktmMemoryStats.argtypes = [C.POINTER(C.c_ulonglong), C.POINTER(C.c_size_t),
                                 C.POINTER(C.c_size_t)]
    L.ktmMemoryStats.restype = C.c_int
    L.ktmCheckDeviceWaits.argtypes = []
    L.ktmCheckDeviceWaits.restype = C.c_int
    L.ktmSelfTestDeviceWait.argtypes = [C.c_int, C.c_int]
    L.ktmSelfTestDeviceWait.restype = C.c_int
    if L.ktmJobStructSize() != C.sizeof(KtmJob):
        raise KtmError(-1, f"ktm_job layout mismatch: library {L.ktmJobStructSize()} bytes, "
                           f"binding {C.sizeof(KtmJob)} bytes")
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != KTM_OK:
        L = lib()
        raise KtmError(rc, L.ktmGetLastErrorMessage().decode(errors="replace")
                       or L.ktmGetErrorString(rc).decode())


def memory_stats() -> dict:
    """The library's own device memory pool (ktmMemoryStats): allocations made
    since it loaded, and the current device's reserved / used bytes."""
    n, r, u = C.c_ulonglong(), C.c_size_t(), C.c_size_t()
    check(lib().ktmMemoryStats(C.byref(n), C.byref(r), C.byref(u)))
    return {"allocations": int(n.value), "reserved": int(r.value), "used": int(u.value)}


def last_error() -> tuple[int, str]:
    L = lib()
    return L.ktmGetLastError(), L.ktmGetLastErrorMessage().decode(errors="replace")
