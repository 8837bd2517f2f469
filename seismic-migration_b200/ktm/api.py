"""Python mirror of the reference's PSTM interface over libktm.so.

``ktmMigrationCPU`` / ``ktmMigrationGPU`` keep the argument list of
psktmCPU.c:13-23 (grids, config, mid/off vectors, traces, velocity, image);
``migrate`` is the extended job (``ktmMigrate`` in include/ktm.h).  Arrays are
numpy (host memory: the library copies in and out) or CUDA torch tensors
(device memory: the call is asynchronous on the given stream).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import ImageGrid, JobParams, KtmError, KtmJob, check, lib

_PICK = {"truncate": _lib.KTM_PICK_TRUNCATE, "linear": _lib.KTM_PICK_LINEAR}
_MODE = {"reference": _lib.KTM_MODE_REFERENCE, "fast": _lib.KTM_MODE_FAST}
_FMT = {"f32": _lib.KTM_FMT_F32, "f16": _lib.KTM_FMT_F16, "bf16": _lib.KTM_FMT_BF16,
        "ibm32": _lib.KTM_FMT_IBM32, "f64": _lib.KTM_FMT_F64}


def grid(n: int, step: float, start: float = 0.0) -> ImageGrid:
    return ImageGrid(int(n), float(step), float(start))


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def as_grid(g) -> ImageGrid:
    """Any object with imagePnts / imageStep / imageStart (or a 3-tuple)."""
    if isinstance(g, ImageGrid):
        return g
    if isinstance(g, (tuple, list)):
        return ImageGrid(int(g[0]), float(g[1]), float(g[2]))
    return ImageGrid(int(g.imagePnts), float(g.imageStep), float(g.imageStart))


def as_params(c) -> JobParams:
    if isinstance(c, JobParams):
        return c
    if isinstance(c, (tuple, list)):
        return JobParams(int(c[0]), int(c[1]), float(c[2]))
    return JobParams(int(c.traceNo), int(c.tracePts), float(c.traceSampleRate))


def _dropin(fn, imageX, imageY, imageZ, config, midX, midY, offX, offY, traces, slowness,
            image=None) -> np.ndarray:
    midX, midY, offX, offY, traces, slowness = map(_f32, (midX, midY, offX, offY, traces,
                                                          slowness))
    imageX, imageY, imageZ = map(as_grid, (imageX, imageY, imageZ))
    config = as_params(config)
    shape = (imageX.imagePnts, imageY.imagePnts, imageZ.imagePnts)
    if image is None:
        image = np.empty(shape, np.float32)
    if image.dtype != np.float32 or not image.flags.c_contiguous or image.size != np.prod(shape):
        raise ValueError("image must be a contiguous float32 array of Nx*Ny*Nz values")
    if traces.size < config.traceNo * config.tracePts:
        raise ValueError("traces holds fewer than traceNo*tracePts samples")
    L = lib()
    getattr(L, fn)(C.byref(imageX), C.byref(imageY), C.byref(imageZ), C.byref(config),
                   midX.ctypes.data, midY.ctypes.data, offX.ctypes.data, offY.ctypes.data,
                   traces.ctypes.data, slowness.ctypes.data, image.ctypes.data)
    code, msg = _lib.last_error()
    if code:
        raise KtmError(code, msg)
    return image


def ktmMigrationCPU(imageX, imageY, imageZ, config, midX, midY, offX, offY, traces, slowness,
                    image=None) -> np.ndarray:
    """psktmCPU.c:13-23 on the GPU: bit-identical image, overwritten."""
    return _dropin("ktmMigrationCPU", imageX, imageY, imageZ, config, midX, midY, offX, offY,
                   traces, slowness, image)


def ktmMigrationGPU(imageX, imageY, imageZ, config, midX, midY, offX, offY, traces, slowness,
                    image=None) -> np.ndarray:
    """psktmCUDA.cu:211-221 signature; same result as ktmMigrationCPU."""
    return _dropin("ktmMigrationGPU", imageX, imageY, imageZ, config, midX, midY, offX, offY,
                   traces, slowness, image)


def initThreeAxes(imageX, imageY, imageZ):
    imageX, imageY, imageZ = map(as_grid, (imageX, imageY, imageZ))
    xx = np.empty(imageX.imagePnts, np.float32)
    yy = np.empty(imageY.imagePnts, np.float32)
    zz = np.empty(imageZ.imagePnts, np.float32)
    lib().initThreeAxes(C.byref(imageX), C.byref(imageY), C.byref(imageZ), xx.ctypes.data,
                        yy.ctypes.data, zz.ctypes.data)
    return xx, yy, zz


# ------------------------------------------------------------------------------------------
def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _ptr(a):
    if a is None:
        return None
    if _is_torch(a):
        return a.data_ptr()
    return a.ctypes.data


def _stream_handle(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


_RHO = {None: 0, 0: 0, "none": 0, 1: 1, "2d": 1, 2: 2, "2.5d": 2, 3: 3, "3d": 3}


class PackedTraces:
    """A packed trace set from ``prepare`` (ktmPrepareTraces): CUDA tensor
    [traceNo, pitch] of F32/F16/BF16 with zero guard samples, a per-trace FP32
    scale, and whether sqrt(j*dt) is folded into the samples."""

    def __init__(self, data, scale, nt: int, fmt: str, prefolded: bool, rho: int):
        self.data, self.scale, self.nt, self.fmt = data, scale, int(nt), fmt
        self.prefolded, self.rho = bool(prefolded), int(rho)

    @property
    def pitch(self) -> int:
        return int(self.data.shape[1])

    @property
    def ntr(self) -> int:
        return int(self.data.shape[0])

    def unpacked(self):
        """float32 [traceNo, nt]: scale * samples (guards dropped)."""
        return self.data[:, : self.nt].float() * self.scale[:, None]


def packed_pitch(nt: int, fmt: str = "bf16") -> int:
    return int(lib().ktmPackedPitch(int(nt), _FMT[fmt]))


def prepare(traces, dt: float, *, fmt: str = "bf16", rho=0, prefold: bool = True,
            script_order: bool = False, stream=None, out=None, out_scale=None,
            nt=None) -> PackedTraces:
    """Rho filter (ktmApplyRhoFilter.m option 1/2/3), sqrt(t) weight fold,
    per-trace scale and quantisation on the device (ktmPrepareTraces).  An
    int32/uint32 tensor holds IBM-32 words, converted in the same pass.
    ``nt``: the first nt samples of each row are the trace (rows of a packed
    set, for instance); default the row length."""
    import torch
    ibm = _is_torch(traces) and traces.dtype in (torch.int32, torch.uint32)
    if not (_is_torch(traces) and traces.is_cuda and (traces.dtype == torch.float32 or ibm)):
        raise ValueError("prepare takes a CUDA float32 (or IBM-32 int32) tensor "
                         "[traceNo, tracePts]")
    traces = traces.contiguous()
    ntr, stride = traces.shape
    nt = stride if nt is None else int(nt)
    if not 0 < nt <= stride:
        raise ValueError("nt must be in 1..row length")
    pitch = packed_pitch(nt, fmt)
    dtype = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[fmt]
    if out is None:
        out = torch.empty((ntr, pitch), device=traces.device, dtype=dtype)
    if out_scale is None:
        out_scale = torch.empty(ntr, device=traces.device, dtype=torch.float32)
    p = _lib.KtmPrep()
    p.traceNo, p.tracePts, p.inStride, p.sampleRate = ntr, nt, stride, float(dt)
    p.in_ = traces.data_ptr()
    p.rho = _RHO[rho if not isinstance(rho, str) else rho.lower()]
    p.rhoScriptOrder = int(bool(script_order))
    p.prefold = int(bool(prefold))
    p.outFormat = _FMT[fmt]
    p.outPitch = int(out.shape[1])
    p.out = out.data_ptr()
    p.outScale = out_scale.data_ptr()
    p.stream = _stream_handle(stream)
    p.inFormat = _lib.KTM_FMT_IBM32 if ibm else _lib.KTM_FMT_F32
    check(lib().ktmPrepareTraces(C.byref(p)))
    return PackedTraces(out, out_scale, nt, fmt, prefold, p.rho)


class Job:
    """Builds a ktm_job and keeps every array it points at alive."""

    def __init__(self, *, imageX, imageY, imageZ, dt, midX, midY, offX, offY, traces,
                 velocity, image=None, scale=None, mode="fast", pick="linear",
                 aperture=0.0, accumulate=False, prefolded=False, fmt=None, stream=None,
                 tile_run=0, pairs_counter=None, trace_stride=0, rho=0, pack_format="f32",
                 weight="table", tile_cols=0, tile_chunk=0, tile=None):
        packed = None
        if isinstance(traces, PackedTraces):
            packed = traces
            traces, scale, fmt = packed.data, packed.scale, packed.fmt
            prefolded, trace_stride = packed.prefolded, packed.pitch
        dev = _is_torch(traces)
        self.device = dev
        imageX, imageY, imageZ = map(as_grid, (imageX, imageY, imageZ))
        self.keep = []
        nx, ny, nz = imageX.imagePnts, imageY.imagePnts, imageZ.imagePnts
        if dev:
            import torch
            if not traces.is_cuda:
                raise ValueError("torch tensors must be CUDA tensors")
            ntr = traces.shape[0]
            nt = packed.nt if packed is not None else traces.shape[1]
            if fmt is None:
                fmt = {torch.float32: "f32", torch.float16: "f16", torch.bfloat16: "bf16",
                       torch.int32: "ibm32", torch.uint32: "ibm32",
                       torch.float64: "f64"}[traces.dtype]
            if image is None:
                image = torch.empty((nx, ny, nz), device=traces.device, dtype=torch.float32)
            for a in (midX, midY, offX, offY, velocity, image, scale):
                if a is not None and not a.is_contiguous():
                    raise ValueError("device arrays must be contiguous")
        else:
            traces = np.ascontiguousarray(traces)
            if fmt is None:
                fmt = {np.dtype(np.float32): "f32", np.dtype(np.float16): "f16",
                       np.dtype(np.uint32): "ibm32"}.get(traces.dtype, "f32")
                if fmt == "f32":
                    traces = _f32(traces)
            midX, midY, offX, offY, velocity = map(_f32, (midX, midY, offX, offY, velocity))
            if scale is not None:
                scale = _f32(scale)
            if image is None:
                image = np.zeros((nx, ny, nz), np.float32)
            ntr = traces.shape[0]
            nt = traces.shape[1]
        self.image = image
        self.keep += [midX, midY, offX, offY, traces, velocity, image, scale]
        j = KtmJob()
        lib().ktmJobInit(C.byref(j))
        j.imageX, j.imageY, j.imageZ = imageX, imageY, imageZ
        j.config = JobParams(int(ntr), int(nt), float(dt))
        j.midX, j.midY, j.offX, j.offY = map(_ptr, (midX, midY, offX, offY))
        j.traces = _ptr(traces)
        j.traceScale = _ptr(scale)
        j.traceFormat = _FMT[fmt]
        j.traceStride = int(trace_stride)
        j.tracesPacked = int(packed is not None)
        j.tracesPrefolded = int(bool(prefolded))
        j.velocity = _ptr(velocity)
        j.velocityCube = int(len(velocity.shape) == 3)
        j.image = _ptr(image)
        j.mode = _MODE[mode]
        j.pick = _PICK[pick]
        j.aperture = float(aperture)
        j.accumulate = int(bool(accumulate))
        j.deviceMemory = int(dev)
        j.stream = _stream_handle(stream)
        if tile is not None:                 # a shape from autotune_tile (dict or KtmTile)
            get = tile.get if isinstance(tile, dict) else lambda k: getattr(tile, k)
            tile_run, tile_cols, tile_chunk = get("tileRun"), get("tileCols"), get("tileChunk")
        j.tileRun = int(tile_run)
        j.tileCols = int(tile_cols)
        j.tileChunk = int(tile_chunk)
        j.pairsEvaluated = _ptr(pairs_counter)
        j.rho = _RHO[rho if not isinstance(rho, str) else rho.lower()]
        j.packFormat = _FMT[pack_format]
        j.weightMethod = {"table": 0, "sqrt": 1, "prefold": 2}[weight]
        self.job = j

    def run(self):
        check(lib().ktmMigrate(C.byref(self.job)))
        return self.image


def migrate(**kw):
    """One migration (ktmMigrate).  Returns the image array / tensor."""
    return Job(**kw).run()


def migrate_batch(jobs, stream=None):
    """Many jobs in one persistent launch (ktmMigrateBatch).  ``jobs`` is a list
    of keyword dicts as for ``migrate`` (device memory, packed traces, images
    given).  Returns the list of images."""
    built = [Job(**kw) for kw in jobs]
    arr = (KtmJob * len(built))(*[b.job for b in built])
    check(lib().ktmMigrateBatch(arr, len(built), _stream_handle(stream)))
    return [b.image for b in built]


def autotune(**kw) -> int:
    """The tau run (tileRun) of the fastest tile for this job's shapes (ktmAutotune)."""
    job = Job(**kw)
    out = C.c_int(0)
    check(lib().ktmAutotune(C.byref(job.job), C.byref(out)))
    return int(out.value)


def autotune_tile(**kw) -> dict:
    """The fastest tile shape for this job (ktmAutotuneTile): tileRun, tileCols,
    tileChunk, ctasPerSm and the measured ms; pass it back as ``tile=``."""
    job = Job(**kw)
    t = _lib.KtmTile()
    check(lib().ktmAutotuneTile(C.byref(job.job), C.byref(t)))
    return t.as_dict()


def tile_candidates(**kw) -> list[dict]:
    """Every tile shape ktmAutotuneTile times for this job (ktmTileCandidates)."""
    job = Job(**kw)
    n = C.c_int(0)
    check(lib().ktmTileCandidates(C.byref(job.job), None, 0, C.byref(n)))
    arr = (_lib.KtmTile * max(1, n.value))()
    check(lib().ktmTileCandidates(C.byref(job.job), arr, n.value, C.byref(n)))
    return [arr[i].as_dict() for i in range(n.value)]


def migrate_columns_f64(*, columns=None, ncols=None, **kw):
    """FP64 device evaluation for a list of image columns -> torch float64 [ncols, Nz]."""
    import torch
    job = Job(**kw)
    if not job.device:
        raise ValueError("migrate_columns_f64 takes CUDA tensors")
    nz = kw["imageZ"].imagePnts
    if columns is not None:
        cols = columns.to(device=kw["midX"].device, dtype=torch.int32).contiguous()
        n = cols.numel()
    else:
        cols, n = None, int(ncols)
    out = torch.empty((n, nz), device=kw["midX"].device, dtype=torch.float64)
    check(lib().ktmMigrateColumnsF64(C.byref(job.job), _ptr(cols), int(n), out.data_ptr()))
    return out


def interp_time(traces, levels: int, stream=None, out=None):
    """Time-axis interpolation by 2^levels (ktmInterpTraces, ktmInterpTraceBlock.m
    opt 2): CUDA float32 [traceNo, tracePts] -> [traceNo, (tracePts-1) 2^levels + 1],
    the new sample interval dt / 2^levels."""
    import torch
    if not (_is_torch(traces) and traces.is_cuda and traces.dtype == torch.float32):
        raise ValueError("interp_time takes a CUDA float32 tensor [traceNo, tracePts]")
    traces = traces.contiguous()
    ntr, nt = traces.shape
    nout = int(lib().ktmInterpLength(int(nt), int(levels)))
    if out is None:
        out = torch.empty((ntr, nout), device=traces.device, dtype=torch.float32)
    p = _lib.KtmInterp()
    p.traceNo, p.tracePts, p.levels = int(ntr), int(nt), int(levels)
    p.in_, p.inStride = traces.data_ptr(), int(nt)
    p.out, p.outStride = out.data_ptr(), int(out.stride(0))
    p.stream = _stream_handle(stream)
    check(lib().ktmInterpTraces(C.byref(p)))
    return out
