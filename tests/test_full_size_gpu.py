"""Parity at the benchmark configurations' full sizes (needs a B200).

* config 1 in full (256 CMPs x 64 offsets = 16,384 traces of 1001 samples,
  256 x 1001 image, 4.2e9 pairs): the reference-mode drop-in is bit-identical
  to the reference's own psktmCPU.c run with one thread (oracle/_ref; the
  oracle restatement where the reference was not built);
* one full 62,500-trace step of config 2 (200 x 200 x 1501 image, 3.75e12
  pairs) through the fast path: linearity in the data and invariance to
  splitting the traces into accumulated parts, to FP32 rounding -- size-
  independent properties where no oracle finishes in seconds;
* config 3 on that step: the 3-D batch in FP16 and BF16 (per-trace scale, the
  3-D rho filter on the device, sqrt(j dt) folded in) against an FP64 pipeline
  from the same raw traces -- the FP64 rho filter (bench.rho_filter_f64,
  pinned to oracle/rho.py on the CPU) and the FP64 device migration -- on a
  seeded subgrid of columns, within 1e-3.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from test_parity_gpu import rel_l2

pytestmark = pytest.mark.gpu


def test_config1_reference_mode_bit_identical_in_full(cuda, ktm_lib):
    import ktm
    from ktm import synth
    sv = synth.config1()
    tr = synth.synthesize(sv)
    gx, gy, gz = (oracle.grid(a.imagePnts, a.imageStep, a.imageStart)
                  for a in (sv.imageX, sv.imageY, sv.imageZ))
    args = (gx, gy, gz, sv.dt, sv.midX, sv.midY, sv.offX, sv.offY, tr, sv.velocity1d)
    gpu = ktm.ktmMigrationGPU(gx, gy, gz, (sv.ntr, sv.nt, sv.dt), *args[4:])
    if oracle.ref_available():
        cpu = oracle.migrate_reference_c(*args, threads=1)
    else:
        cpu = oracle.migrate_ref32(*args)
    assert np.abs(cpu).max() > 0
    assert np.array_equal(np.asarray(gpu).view(np.uint32), cpu.view(np.uint32))


def test_config2_step_linearity_and_split(cuda, ktm_lib):
    import torch

    import ktm
    from ktm import synth
    dev = cuda
    sv = synth.config2(ntr=62_500, seed=2)
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x)).to(dev)  # noqa: E731
    co = [T(x) for x in (sv.midX, sv.midY, sv.offX, sv.offY)]
    d1 = synth.synthesize_device(sv, device=dev, coords=co)
    d2 = torch.roll(d1, shifts=7, dims=1) * 0.5 - 0.1 * d1
    kw = dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt, midX=co[0],
              midY=co[1], offX=co[2], offY=co[3], velocity=T(sv.velocity), pick="linear",
              aperture=sv.aperture)

    def mig(d, **extra):
        p = ktm.prepare(d, sv.dt, fmt="f32", rho=0, prefold=True)
        return ktm.migrate(traces=p, **kw, **extra)

    i1 = mig(d1).clone()
    i2 = mig(d2).clone()
    i12 = mig(d1 + 2.0 * d2).clone()
    assert float(i1.abs().max()) > 0
    assert rel_l2(i12.cpu().numpy(), (i1 + 2.0 * i2).cpu().numpy()) < 1e-5
    # the traces in two parts, the second accumulated into the first's image
    k = 27_001
    p = ktm.prepare(d1, sv.dt, fmt="f32", rho=0, prefold=True)
    img = torch.empty_like(i1)
    part = lambda s, **e: ktm.migrate(  # noqa: E731
        traces=ktm.PackedTraces(p.data[s], p.scale[s], p.nt, p.fmt, p.prefolded, p.rho),
        **dict(kw, midX=co[0][s], midY=co[1][s], offX=co[2][s], offY=co[3][s]), **e)
    part(slice(0, k), image=img)
    part(slice(k, None), image=img, accumulate=True)
    assert rel_l2(img.cpu().numpy(), i1.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("fmt", ["f16", "bf16"])
def test_config3_mixed_precision_whole_image(cuda, ktm_lib, fmt):
    """Config 3: config 1 with FP16 / BF16 traces (per-trace FP32 scale), 2.5-D rho,
    sqrt(j dt) folded in, against the FP64 device evaluation of the whole image:
    within the 1e-3 relative L2 gate."""
    import torch

    import ktm
    from ktm import synth
    sv = synth.config1()
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x, dtype=np.float32)).to(cuda)  # noqa: E731
    co = [T(x) for x in (sv.midX, sv.midY, sv.offX, sv.offY)]
    raw = synth.synthesize_device(sv, device=cuda, coords=co)
    geo = dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt, midX=co[0],
               midY=co[1], offX=co[2], offY=co[3], velocity=T(sv.velocity1d),
               aperture=sv.aperture, pick="linear")
    p32 = ktm.prepare(raw, sv.dt, fmt="f32", rho=sv.rho_opt, prefold=False)
    nx, ny, nz = sv.shape
    ref = ktm.migrate_columns_f64(ncols=nx * ny, traces=p32, **geo).double()
    p = ktm.prepare(raw, sv.dt, fmt=fmt, rho=sv.rho_opt, prefold=True)
    got = ktm.migrate(traces=p, **geo).reshape(nx * ny, nz).double()
    err = float((got - ref).norm() / ref.norm())
    assert err < 1e-3, err


@pytest.mark.parametrize("fmt", ["f16", "bf16"])
def test_config3_on_the_3d_step_within_1e3_of_the_fp64_pipeline(cuda, ktm_lib, fmt):
    import os
    import sys

    import torch

    import ktm
    from ktm import synth
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    import bench
    sv = synth.config2(ntr=62_500, seed=2)
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x)).to(cuda)  # noqa: E731
    co = [T(x) for x in (sv.midX, sv.midY, sv.offX, sv.offY)]
    raw = synth.synthesize_device(sv, device=cuda, coords=co)
    geo = dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt, midX=co[0],
               midY=co[1], offX=co[2], offY=co[3], velocity=T(sv.velocity), pick="linear",
               aperture=sv.aperture)
    p = ktm.prepare(raw, sv.dt, fmt=fmt, rho=sv.rho_opt, prefold=True)
    img = ktm.migrate(traces=p, weight="prefold", **geo)
    nx, ny, nz = sv.shape
    rng = np.random.default_rng(23)
    cols = torch.as_tensor(np.sort(rng.choice(nx * ny, size=256, replace=False)).astype(np.int32))
    f64 = bench.rho_filter_f64(raw, sv.dt, sv.rho_opt)
    ref = ktm.migrate_columns_f64(columns=cols, traces=f64, **geo).double()
    got = img.reshape(nx * ny, nz)[cols.to(cuda).long()].double()
    err = float((got - ref).norm() / ref.norm())
    assert err < 1e-3, err
