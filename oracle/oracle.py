"""ctypes front end of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module, and only as the checker.  Nothing under the product
package imports it.

Two libraries:
  * ``oracle/libktm_oracle.so`` -- this project's C restatement
    (``ktm_oracle.c``): ``migrate_ref32`` restates psktmCPU.c:13-101
    bit-for-bit; ``migrate_f64`` / ``demigrate_f64`` / ``vrms_grad_f64`` are the
    FP64 extended method.
  * ``oracle/_ref/libktm_ref.so`` -- the reference's own psktmCPU.c,
    psktmFunctions.c and ioFunctions.c compiled unmodified (``oracle/Makefile``),
    present wherever it was built (it travels with the repository snapshot).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libktm_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libktm_ref.so")


class ImageGrid(C.Structure):
    _fields_ = [("imagePnts", C.c_int), ("imageStep", C.c_float), ("imageStart", C.c_float)]


class JobParams(C.Structure):
    _fields_ = [("traceNo", C.c_int), ("tracePts", C.c_int), ("traceSampleRate", C.c_float)]


class OracleJob(C.Structure):
    _fields_ = [
        ("imageX", ImageGrid), ("imageY", ImageGrid), ("imageZ", ImageGrid),
        ("traceNo", C.c_int), ("tracePts", C.c_int), ("traceStride", C.c_int),
        ("sampleRate", C.c_double),
        ("midX", C.c_void_p), ("midY", C.c_void_p), ("offX", C.c_void_p), ("offY", C.c_void_p),
        ("traces", C.c_void_p), ("traceScale", C.c_void_p),
        ("velocity", C.c_void_p), ("velocityCube", C.c_int),
        ("pick", C.c_int), ("aperture", C.c_double), ("prefold", C.c_int),
    ]


def build(quiet: bool = True) -> None:
    """Compile the oracle (and the reference library when its sources exist)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


_lib = None
_ref = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        _lib = C.CDLL(ORACLE_SO)
        P = C.c_void_p
        _lib.oracle_migrate_ref32.argtypes = [P] * 11
        _lib.oracle_migrate_f64.argtypes = [P, P, C.c_int, C.c_int]
        _lib.oracle_demigrate_f64.argtypes = [P, P, P]
        _lib.oracle_vrms_grad_f64.argtypes = [P, P]
        _lib.oracle_count_aperture_pairs.argtypes = [P]
        _lib.oracle_count_aperture_pairs.restype = C.c_ulonglong
        _lib.oracle_ibm32_to_ieee.argtypes = [P, P, C.c_int]
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib() -> C.CDLL:
    """The reference's own compiled psktmCPU.c (raises if it was never built)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO + " not built (reference sources absent)")
        _ref = C.CDLL(REF_SO)
        P = C.c_void_p
        _ref.ktmMigrationCPU.argtypes = [P] * 11
        _ref.ktmMigrationCPU.restype = None
        _ref.ktmIBM32toIEEE.argtypes = [P, P, C.c_int]
        _ref.ktmIBM32toIEEE.restype = None
    return _ref


def set_omp_threads(n: int) -> None:
    """Thread count of the OpenMP runtime the reference library uses."""
    ref_lib()
    gomp = C.CDLL("libgomp.so.1")
    gomp.omp_set_num_threads(C.c_int(int(n)))


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def grid(n: int, step: float, start: float) -> ImageGrid:
    return ImageGrid(int(n), float(step), float(start))


def _ref_args(gx, gy, gz, ntr, nt, dt, midx, midy, offx, offy, traces, vel, image):
    gx, gy, gz = _as_grid(gx), _as_grid(gy), _as_grid(gz)
    cfg = JobParams(int(ntr), int(nt), float(dt))
    return [C.byref(gx), C.byref(gy), C.byref(gz), C.byref(cfg),
            _p(midx), _p(midy), _p(offx), _p(offy), _p(traces), _p(vel), _p(image)]


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def migrate_ref32(gx, gy, gz, dt, midx, midy, offx, offy, traces, vel) -> np.ndarray:
    """Restatement of psktmCPU.c (bit-identical to it with one thread)."""
    midx, midy, offx, offy, traces, vel = map(_f32, (midx, midy, offx, offy, traces, vel))
    ntr, nt = traces.shape
    image = np.empty((gx.imagePnts, gy.imagePnts, gz.imagePnts), np.float32)
    args = _ref_args(gx, gy, gz, ntr, nt, dt, midx, midy, offx, offy, traces, vel, image)
    # keep the JobParams alive through the call
    lib().oracle_migrate_ref32(*args)
    return image


def migrate_reference_c(gx, gy, gz, dt, midx, midy, offx, offy, traces, vel,
                        threads: int = 1) -> np.ndarray:
    """The reference's own ktmMigrationCPU (compiled unmodified)."""
    midx, midy, offx, offy, traces, vel = map(_f32, (midx, midy, offx, offy, traces, vel))
    ntr, nt = traces.shape
    image = np.empty((gx.imagePnts, gy.imagePnts, gz.imagePnts), np.float32)
    set_omp_threads(threads)
    args = _ref_args(gx, gy, gz, ntr, nt, dt, midx, midy, offx, offy, traces, vel, image)
    ref_lib().ktmMigrationCPU(*args)
    return image


def _as_grid(g) -> ImageGrid:
    """Any object with imagePnts / imageStep / imageStart (e.g. the product's own grid)."""
    if isinstance(g, ImageGrid):
        return g
    return ImageGrid(int(g.imagePnts), float(g.imageStep), float(g.imageStart))


class _Job:
    """Holds an OracleJob and the arrays it points at."""

    def __init__(self, gx, gy, gz, dt, midx, midy, offx, offy, traces, vel, *,
                 scale=None, pick=1, aperture=0.0, prefold=False):
        gx, gy, gz = _as_grid(gx), _as_grid(gy), _as_grid(gz)
        self.keep = [_f32(a) for a in (midx, midy, offx, offy, traces, vel)]
        midx, midy, offx, offy, traces, vel = self.keep
        if scale is not None:
            scale = _f32(scale)
            self.keep.append(scale)
        ntr, nt = traces.shape
        cube = vel.ndim == 3
        # the library takes the sample interval as a float (jobParams.traceSampleRate)
        self.job = OracleJob(
            gx, gy, gz, ntr, nt, nt, float(np.float32(dt)),
            _p(midx), _p(midy), _p(offx), _p(offy), _p(traces),
            _p(scale) if scale is not None else None,
            _p(vel), int(cube), int(pick), float(aperture), int(prefold))
        self.shape = (gx.imagePnts, gy.imagePnts, gz.imagePnts)
        self.ntr, self.nt = ntr, nt


def migrate_f64(gx, gy, gz, dt, midx, midy, offx, offy, traces, vel, *, scale=None,
                pick=1, aperture=0.0, prefold=False, columns=None) -> np.ndarray:
    """FP64 extended-method oracle.  ``columns`` = (col0, ncol) restricts the
    output to a contiguous run of image columns (returned as [ncol, Nz])."""
    j = _Job(gx, gy, gz, dt, midx, midy, offx, offy, traces, vel, scale=scale,
             pick=pick, aperture=aperture, prefold=prefold)
    if columns is None:
        out = np.empty(j.shape, np.float64)
        lib().oracle_migrate_f64(C.byref(j.job), _p(out), 0, 0)
    else:
        c0, nc = columns
        out = np.empty((nc, j.shape[2]), np.float64)
        lib().oracle_migrate_f64(C.byref(j.job), _p(out), int(c0), int(nc))
    return out


def demigrate_f64(gx, gy, gz, dt, midx, midy, offx, offy, nt, vel, image, *, pick=1,
                  aperture=0.0, prefold=False) -> np.ndarray:
    """Exact transpose of ``migrate_f64`` -> data [traceNo, nt]."""
    ntr = len(midx)
    dummy = np.zeros((ntr, nt), np.float32)
    j = _Job(gx, gy, gz, dt, midx, midy, offx, offy, dummy, vel, pick=pick,
             aperture=aperture, prefold=prefold)
    img = np.ascontiguousarray(image, dtype=np.float64)
    out = np.empty((ntr, nt), np.float64)
    lib().oracle_demigrate_f64(C.byref(j.job), _p(img), _p(out))
    return out


def vrms_grad_f64(gx, gy, gz, dt, midx, midy, offx, offy, traces, vel, *, aperture=0.0,
                  prefold=False) -> np.ndarray:
    """dI[p]/dv[p] (velocity-cube semantics, linear pick), FP64."""
    j = _Job(gx, gy, gz, dt, midx, midy, offx, offy, traces, vel, pick=1,
             aperture=aperture, prefold=prefold)
    out = np.empty(j.shape, np.float64)
    lib().oracle_vrms_grad_f64(C.byref(j.job), _p(out))
    return out


def count_aperture_pairs(gx, gy, gz, midx, midy, aperture: float) -> int:
    n = len(midx)
    z = np.zeros(n, np.float32)
    j = _Job(gx, gy, gz, 1.0, midx, midy, z, z, np.zeros((n, 1), np.float32),
             np.ones(gz.imagePnts, np.float32), aperture=aperture)
    return int(lib().oracle_count_aperture_pairs(C.byref(j.job)))


def ibm32_to_ieee(words: np.ndarray) -> np.ndarray:
    w = np.ascontiguousarray(words, dtype=np.uint32)
    out = np.empty(w.shape, np.float32)
    lib().oracle_ibm32_to_ieee(_p(w), _p(out), int(w.size))
    return out


def ibm32_to_ieee_reference_c(words: np.ndarray) -> np.ndarray:
    w = np.ascontiguousarray(words, dtype=np.uint32)
    out = np.empty(w.shape, np.float32)
    ref_lib().ktmIBM32toIEEE(_p(w), _p(out), int(w.size))
    return out
