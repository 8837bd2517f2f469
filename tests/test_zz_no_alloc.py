"""ktmMigratePackedNoAlloc: the migration entry point for callers that cannot
allocate device memory while they run (a loop that must never let an
allocation synchronise the GPU, or a framework that has already divided the
GPU's memory among its own pools).  Its scratch is a static 16 MiB device array
instead of an allocation.

Checked through the C ABI against ktmMigrate on the same packed traces, twice in
a row (the array keeps the previous call's contents), for the cases that stress
the array: the prefolded weight, an image of 1.5 Mi samples (two partial images
fill the array), a trace set that goes in several launches (the array reused
within one call) and accumulation.  The library's allocation counter must not
move during the calls.  This file is named to be collected last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(dev, *, ntr=3000, nt=400, shape=(24, 3, 350), fmt="f16", prefold=False, seed=31):
    import torch

    import ktm
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    gx, gy = ktm.grid(nx, 25.0, -12.5 * nx), ktm.grid(ny, 25.0, -12.5 * ny)
    gz = ktm.grid(nz, 0.002, 0.0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(dev)  # noqa: E731
    mid = rng.uniform(-500.0, 500.0, (ntr, 2))
    off = rng.uniform(-400.0, 400.0, (ntr, 2))
    traces = t(rng.standard_normal((ntr, nt)))
    packed = ktm.prepare(traces, 0.004, fmt=fmt, prefold=prefold)
    vel = t(np.linspace(1500.0, 3200.0, nz))
    kw = dict(imageX=gx, imageY=gy, imageZ=gz, dt=0.004, midX=t(mid[:, 0]), midY=t(mid[:, 1]),
              offX=t(off[:, 0]), offY=t(off[:, 1]), traces=packed, velocity=vel,
              pick="linear", aperture=600.0, weight="prefold" if prefold else "table")
    return kw


def _rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _check_twice(kw, start=None):
    """Two no-allocation calls in a row against ktmMigrate; returns nothing, asserts."""
    import torch

    import ktm
    from ktm import _lib
    L = ktm.lib()
    acc = start is not None
    ref_img = start.clone() if acc else None
    expect = ktm.migrate(image=ref_img, accumulate=acc, **kw).cpu().numpy()   # allocating entry
    assert np.abs(expect).max() > 0
    for call in range(2):
        # NaN where nothing accumulates: every sample must be written
        out = start.clone() if acc else torch.full(expect.shape, float("nan"),
                                                   device=kw["midX"].device)
        job = ktm.Job(image=out, accumulate=acc, **kw)
        torch.cuda.synchronize()
        before = _lib.memory_stats()["allocations"]
        rc = L.ktmMigratePackedNoAlloc(C.byref(job.job))
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert _lib.memory_stats()["allocations"] == before, f"call {call} allocated"
        got = out.cpu().numpy()
        assert np.isfinite(got).all(), f"call {call}"
        # same kernel, different trace-slice count: only the summation order differs
        assert _rel_l2(got, expect) < 2e-5, f"call {call}"


def test_no_alloc_matches_ktm_migrate_twice(cuda):
    _check_twice(_case(cuda))


def test_no_alloc_prefolded_weight(cuda):
    """KTM_WEIGHT_PREFOLD with samples prepared with prefold = 1 (the benchmark's method)."""
    _check_twice(_case(cuda, prefold=True, seed=32))


def test_no_alloc_image_of_1_5_mi_samples(cuda):
    """1.5 Mi samples: two partial images fill the 4 Mi-float array."""
    _check_twice(_case(cuda, ntr=2000, shape=(40, 40, 983), nt=1000, seed=33))


def test_no_alloc_traces_in_several_launches(cuda):
    """F32 rows of 2008 samples: 40 MB holds ~5200 of them, so 12,000 traces go in three
    launches that reuse the array within one call."""
    _check_twice(_case(cuda, ntr=12000, nt=2000, shape=(8, 4, 300), fmt="f32", seed=34))


def test_no_alloc_accumulates(cuda):
    import torch
    kw = _case(cuda, seed=35)
    g = torch.Generator(device=cuda).manual_seed(7)
    start = torch.randn((24, 3, 350), device=cuda, generator=g)
    _check_twice(kw, start=start)


def test_no_alloc_rejects_images_beyond_its_scratch(cuda):
    import torch

    import ktm
    L = ktm.lib()
    kw = _case(cuda)
    kw["imageZ"] = ktm.grid(2_200_000 // (24 * 3) + 1, 0.002, 0.0)    # > 2 Mi samples
    kw["velocity"] = torch.full((kw["imageZ"].imagePnts,), 2000.0, device=cuda)
    job = ktm.Job(image=torch.empty(1, device=cuda), **kw)
    rc = L.ktmMigratePackedNoAlloc(C.byref(job.job))
    code, msg = ktm._lib.last_error()
    assert rc == ktm._lib.KTM_ERR_LIMIT and code == rc
    assert "exceeds the limit" in msg
