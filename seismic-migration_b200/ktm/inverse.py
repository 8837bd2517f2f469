"""Adjoint, velocity gradient and least-squares migration over the C ABI.

``MigrationOperator`` binds one survey geometry and exposes
  * ``migrate(data)``   -- L^T: packed F32 data [traceNo, pitch] -> image (ktmMigrate)
  * ``demigrate(image)`` -- L: image -> packed F32 data (ktmDemigrate)
which are exact transposes of each other (weight "table", "sqrt" or "prefold":
with "prefold" L^T folds sqrt(j dt) into the data with ktmPrepareTraces and
migrates the folded samples, and L scatters without a per-pair weight and
multiplies each data sample by sqrt(j dt)); ``Migrate`` / ``Demigrate`` wrap them
as ``torch.autograd.Function`` for the tests and the least-squares harness
(autograd does not run inside the library).  ``vrms_gradient`` returns
dI/dv per image sample (ktmVrmsGradient); ``least_squares`` runs CGLS on the
device (ktmLeastSquaresMigrate), optionally replayed from a CUDA graph.

Data-space vectors use the packed F32 layout of ktmPrepareTraces: pitch =
ktmPackedPitch(tracePts, F32) samples per trace, zero guard samples at 0 and
at j >= tracePts.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import KtmLsm, check, lib
from .api import Job, PackedTraces, as_grid, packed_pitch, prepare


class MigrationOperator:
    def __init__(self, *, imageX, imageY, imageZ, dt, nt, midX, midY, offX, offY, velocity,
                 aperture=0.0, pick="linear", weight="table", stream=None):
        import torch
        self.imageX, self.imageY, self.imageZ = map(as_grid, (imageX, imageY, imageZ))
        self.dt, self.nt = float(dt), int(nt)
        self.midX, self.midY, self.offX, self.offY = midX, midY, offX, offY
        self.velocity = velocity
        self.aperture, self.pick, self.weight, self.stream = aperture, pick, weight, stream
        self.device = midX.device
        self.ntr = int(midX.shape[0])
        self.pitch = packed_pitch(self.nt, "f32")
        self.ones = torch.ones(self.ntr, device=self.device, dtype=torch.float32)
        self.shape = (self.imageX.imagePnts, self.imageY.imagePnts, self.imageZ.imagePnts)

    def _job(self, traces, image):
        return Job(imageX=self.imageX, imageY=self.imageY, imageZ=self.imageZ, dt=self.dt,
                   midX=self.midX, midY=self.midY, offX=self.offX, offY=self.offY,
                   traces=traces, velocity=self.velocity, image=image, pick=self.pick,
                   aperture=self.aperture, weight=self.weight, stream=self.stream)

    def pack(self, traces):
        """[traceNo, nt] float32 -> packed F32 [traceNo, pitch] (sample 0 and the tail zero)."""
        import torch
        out = torch.zeros((self.ntr, self.pitch), device=self.device, dtype=torch.float32)
        out[:, 1:self.nt] = traces[:, 1:self.nt]
        return out

    def packed(self, data):
        return PackedTraces(data, self.ones, self.nt, "f32", False, 0)

    def migrate(self, data, image=None):
        """L^T d: packed F32 data -> image [Nx, Ny, Nz]."""
        import torch
        if image is None:
            image = torch.empty(self.shape, device=self.device, dtype=torch.float32)
        if self.weight == "prefold":
            traces = prepare(data.contiguous(), self.dt, fmt="f32", prefold=True, nt=self.nt,
                             stream=self.stream)
        else:
            traces = self.packed(data.contiguous())
        return self._job(traces, image).run()

    def demigrate(self, image, data=None):
        """L m: image -> packed F32 data [traceNo, pitch]."""
        import torch
        if data is None:
            data = torch.empty((self.ntr, self.pitch), device=self.device, dtype=torch.float32)
        image = image.contiguous()
        job = self._job(self.packed(data), image)
        check(lib().ktmDemigrate(C.byref(job.job), data.data_ptr(), self.pitch))
        return data

    def vrms_gradient(self, packed_traces, grad=None):
        """dI[p]/dv[p] for a packed trace set (linear pick, table weight or prefolded)."""
        import torch
        if grad is None:
            grad = torch.empty(self.shape, device=self.device, dtype=torch.float32)
        job = self._job(packed_traces, grad)
        check(lib().ktmVrmsGradient(C.byref(job.job), grad.data_ptr()))
        return grad

    def least_squares(self, data, iterations: int, model=None, use_graph: bool = True):
        """CGLS for min ||L m - d||: returns (model, residual norms, gradient norms)."""
        import torch
        if model is None:
            model = torch.zeros(self.shape, device=self.device, dtype=torch.float32)
        rn = np.zeros(iterations + 1, np.float64)
        gn = np.zeros(iterations + 1, np.float64)
        job = self._job(self.packed(data), model)
        L = KtmLsm()
        L.job = job.job
        L.data = data.data_ptr()
        L.dataPitch = self.pitch
        L.model = model.data_ptr()
        L.iterations = int(iterations)
        L.useGraph = int(bool(use_graph))
        L.residualNorms = rn.ctypes.data
        L.gradientNorms = gn.ctypes.data
        check(lib().ktmLeastSquaresMigrate(C.byref(L)))
        return model, rn, gn


def _autograd():
    import torch

    class Demigrate(torch.autograd.Function):
        """m -> L m; backward applies L^T."""

        @staticmethod
        def forward(ctx, image, op):
            ctx.op = op
            return op.demigrate(image)

        @staticmethod
        def backward(ctx, g):
            return ctx.op.migrate(g.contiguous()), None

    class Migrate(torch.autograd.Function):
        """d -> L^T d; backward applies L."""

        @staticmethod
        def forward(ctx, data, op):
            ctx.op = op
            return op.migrate(data)

        @staticmethod
        def backward(ctx, g):
            return ctx.op.demigrate(g.contiguous()), None

    return Demigrate, Migrate


def demigrate_fn():
    return _autograd()[0]


def migrate_fn():
    return _autograd()[1]


__all__ = ["MigrationOperator", "demigrate_fn", "migrate_fn", "_lib"]
