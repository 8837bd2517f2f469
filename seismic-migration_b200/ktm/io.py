"""The reference's data directory on disk, through libktm.so's C readers.

    inp.txt          tracePts, dt, traceNo, x/y/tau start-step-points
                     (ktmVisualizeOutputFile.m:22-48, ktmWriteTraceBlockConstOffset.m:154-167)
    inputData.bin    traceNo x tracePts IBM-32 words (or float32, the impulse option)
    inputSrcX/Y.bin, inputRecX/Y.bin   float32 [traceNo]
    velModel.bin     float32 [Nz] (ktmWriteVelModel.m:22-23) or [Nx][Ny][Nz]
    outputData.bin   float32 [Nx][Ny][Nz], tau fastest

SEG-Y files (``segy_open``, ``read_segy``, ``load_segy_survey``) replace the
Octave front end ktmGetInputMeta.m / ktmGetInputTrace.m.

``write_survey`` plays the part of the Octave writers for tests and examples;
``load_survey`` is ktmLoadSurvey (ioFunctions.c:94-153 with the coordinate
conversion of ktmConvertXYtoOffMid.m:12); ``ibm32_to_ieee`` is ktmIBM32toIEEE
(ioFunctions.c:4-40) on the GPU.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import ImageGrid, check, lib


@dataclass
class Inp:
    tracePts: int
    sampleRate: float
    traceNo: int
    x: tuple          # (points, step, start)
    y: tuple
    z: tuple

    def _c(self) -> _lib.KtmInp:
        c = _lib.KtmInp()
        c.tracePts, c.sampleRate, c.traceNo = int(self.tracePts), float(self.sampleRate), int(self.traceNo)
        c.x, c.y, c.z = (ImageGrid(int(a[0]), float(a[1]), float(a[2])) for a in (self.x, self.y, self.z))
        return c

    @staticmethod
    def _from(c: _lib.KtmInp) -> "Inp":
        g = lambda a: (int(a.imagePnts), float(a.imageStep), float(a.imageStart))  # noqa: E731
        return Inp(int(c.tracePts), float(c.sampleRate), int(c.traceNo), g(c.x), g(c.y), g(c.z))


def read_inp(path: str) -> Inp:
    c = _lib.KtmInp()
    check(lib().ktmReadInp(os.fsencode(path), C.byref(c)))
    return Inp._from(c)


def write_inp(path: str, inp: Inp) -> None:
    c = inp._c()
    check(lib().ktmWriteInp(os.fsencode(path), C.byref(c)))


@dataclass
class Survey:
    inp: Inp
    traces: np.ndarray        # [traceNo, tracePts] uint32 IBM words or float32
    midX: np.ndarray
    midY: np.ndarray
    offX: np.ndarray
    offY: np.ndarray
    velocity: np.ndarray      # [Nz] or [Nx, Ny, Nz]
    origin: tuple             # (x, y) subtracted when rebased

    @property
    def fmt(self) -> str:
        return "ibm32" if self.traces.dtype == np.uint32 else "f32"

    def grids(self):
        return tuple(ImageGrid(*a) for a in (self.inp.x, self.inp.y, self.inp.z))


def _copy(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype)
    buf = (C.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr)
    return np.frombuffer(buf, dtype=dtype, count=n).copy()


def load_survey(directory: str, ibm: bool = True, rebase: bool = False) -> Survey:
    """Read a data directory (ktmLoadSurvey).  IBM words are returned as read:
    the migration converts them on the device."""
    s = _lib.KtmSurvey()
    check(lib().ktmLoadSurvey(os.fsencode(directory), int(bool(ibm)), int(bool(rebase)), C.byref(s)))
    try:
        inp = Inp._from(s.inp)
        ntr, nt = inp.traceNo, inp.tracePts
        nz = inp.z[0]
        dt = np.uint32 if s.traceFormat == _lib.KTM_FMT_IBM32 else np.float32
        traces = _copy(s.traces, ntr * nt, dt).reshape(ntr, nt)
        co = [_copy(getattr(s, f), ntr, np.float32) for f in ("midX", "midY", "offX", "offY")]
        if s.velocityCube:
            vel = _copy(s.velocity, inp.x[0] * inp.y[0] * nz, np.float32).reshape(inp.x[0], inp.y[0], nz)
        else:
            vel = _copy(s.velocity, nz, np.float32)
        return Survey(inp, traces, *co, vel, (float(s.originX), float(s.originY)))
    finally:
        lib().ktmFreeSurvey(C.byref(s))


def write_image(path: str, image) -> None:
    """outputData.bin (ktmWriteImage): float32 [Nx][Ny][Nz]."""
    if type(image).__module__.startswith("torch"):
        image = image.detach().cpu().numpy()
    a = np.ascontiguousarray(image, dtype=np.float32)
    check(lib().ktmWriteImage(os.fsencode(path), a.ctypes.data, a.size))


def read_image(path: str, inp: Inp) -> np.ndarray:
    """outputData.bin as ktmVisualizeOutputFile.m:16-28 reads it."""
    return np.fromfile(path, dtype=np.float32).reshape(inp.x[0], inp.y[0], inp.z[0])


def write_survey(directory: str, inp: Inp, traces, srcX, srcY, recX, recY, velocity) -> None:
    """Write the files the Octave writers produce (ktmWriteTraceBlockConstOffset.m:
    128-167, ktmWriteVelModel.m:22-23): ``traces`` uint32 (IBM-32 words) or float32."""
    os.makedirs(directory, exist_ok=True)
    tr = np.ascontiguousarray(traces)
    if tr.dtype not in (np.uint32, np.float32):
        raise ValueError("traces must be uint32 IBM words or float32")
    tr.tofile(os.path.join(directory, "inputData.bin"))
    for name, a in (("inputSrcX", srcX), ("inputSrcY", srcY), ("inputRecX", recX), ("inputRecY", recY)):
        np.ascontiguousarray(a, dtype=np.float32).tofile(os.path.join(directory, name + ".bin"))
    np.ascontiguousarray(velocity, dtype=np.float32).tofile(os.path.join(directory, "velModel.bin"))
    write_inp(os.path.join(directory, "inp.txt"), inp)


def ibm32_to_ieee(words, stream=None):
    """IBM-32 -> IEEE float on the GPU, bit-identical to ktmIBM32toIEEE.
    numpy uint32 in -> numpy float32 out (host buffers, synchronous); a CUDA
    int32/uint32 tensor in -> float32 tensor out (asynchronous on ``stream``)."""
    if type(words).__module__.startswith("torch"):
        import torch
        if not words.is_cuda or words.dtype not in (torch.int32, torch.uint32):
            raise ValueError("a CUDA int32/uint32 tensor of IBM words is expected")
        w = words.contiguous()
        out = torch.empty(w.shape, device=w.device, dtype=torch.float32)
        h = None if stream is None else (stream if isinstance(stream, int) else stream.cuda_stream)
        check(lib().ktmIBM32toIEEEDevice(w.data_ptr(), out.data_ptr(), w.numel(), h))
        return out
    w = np.ascontiguousarray(words, dtype=np.uint32)
    out = np.empty(w.shape, np.float32)
    if w.size:
        lib().ktmIBM32toIEEE(w.ctypes.data, out.ctypes.data, int(w.size))
        code, msg = _lib.last_error()
        if code:
            raise _lib.KtmError(code, msg)
    return out


# ------------------------------------------------------------------------------ SEG-Y ---
def segy_open(path: str, big_endian: bool = True) -> _lib.KtmSegyInfo:
    """Reel headers of a SEG-Y file (ktmSegyOpen)."""
    info = _lib.KtmSegyInfo()
    check(lib().ktmSegyOpen(os.fsencode(path), int(bool(big_endian)), C.byref(info)))
    return info


def read_segy(path: str, first: int = 0, count: int | None = None, big_endian: bool = True,
              headers: bool = True):
    """Traces [first, first + count) of a SEG-Y file (ktmSegyReadTraces).
    Returns (info, samples, trace headers): samples uint32 IBM words for format 1
    (decoded on the GPU by the migration or ``ibm32_to_ieee``), float32 otherwise;
    headers a list of ``ktm_segy_trace`` (or None)."""
    info = segy_open(path, big_endian)
    if count is None:
        count = int(info.traceCount) - first
    ns = int(info.samplesPerTrace)
    ibm = lib().ktmSegyTraceFormat(C.byref(info)) == _lib.KTM_FMT_IBM32
    samples = np.empty((count, ns), np.uint32 if ibm else np.float32)
    hdr = (_lib.KtmSegyTrace * max(count, 1))() if headers else None
    check(lib().ktmSegyReadTraces(os.fsencode(path), C.byref(info), int(first), int(count),
                                  samples.ctypes.data if count else None, hdr))
    return info, samples, (list(hdr)[:count] if headers else None)


def load_segy_survey(path: str, first: int = 0, count: int = -1, big_endian: bool = True,
                     rebase: bool = False) -> Survey:
    """A survey from a SEG-Y file (ktmLoadSegySurvey).  The image grid and the
    velocity are not in the file: ``inp.x/y/z`` are zero and ``velocity`` is empty."""
    s = _lib.KtmSurvey()
    check(lib().ktmLoadSegySurvey(os.fsencode(path), int(bool(big_endian)), int(first), int(count),
                                  int(bool(rebase)), C.byref(s)))
    try:
        inp = Inp._from(s.inp)
        ntr, nt = inp.traceNo, inp.tracePts
        dt = np.uint32 if s.traceFormat == _lib.KTM_FMT_IBM32 else np.float32
        traces = _copy(s.traces, ntr * nt, dt).reshape(ntr, nt)
        co = [_copy(getattr(s, f), ntr, np.float32) for f in ("midX", "midY", "offX", "offY")]
        return Survey(inp, traces, *co, np.zeros(0, np.float32), (float(s.originX), float(s.originY)))
    finally:
        lib().ktmFreeSurvey(C.byref(s))
