"""ktmMigratePackedNoAlloc: the migration entry point for callers that cannot
allocate device memory while they run (a loop that must never let an
allocation synchronise the GPU, or a framework that has already divided the
GPU's memory among its own pools).  Its scratch is a static 16 MiB device array
instead of an allocation.

Checked through the C ABI against ktmMigrate on the same packed traces, twice in
a row (the array keeps the previous call's contents), plus the size limit.
This file is named to be collected last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(dev):
    import torch

    import ktm
    rng = np.random.default_rng(31)
    ntr, nt = 3000, 400
    gx, gy, gz = ktm.grid(24, 25.0, -300.0), ktm.grid(3, 25.0, -25.0), ktm.grid(350, 0.002, 0.0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(dev)  # noqa: E731
    mid = rng.uniform(-500.0, 500.0, (ntr, 2))
    off = rng.uniform(-400.0, 400.0, (ntr, 2))
    traces = t(rng.standard_normal((ntr, nt)))
    packed = ktm.prepare(traces, 0.004, fmt="f16", prefold=False)
    vel = t(np.linspace(1500.0, 3200.0, gz.imagePnts))
    kw = dict(imageX=gx, imageY=gy, imageZ=gz, dt=0.004, midX=t(mid[:, 0]), midY=t(mid[:, 1]),
              offX=t(off[:, 0]), offY=t(off[:, 1]), traces=packed, velocity=vel,
              pick="linear", aperture=600.0)
    return kw


def _rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_no_alloc_matches_ktm_migrate_twice(cuda):
    import torch

    import ktm
    L = ktm.lib()
    kw = _case(cuda)
    expect = ktm.migrate(**kw).cpu().numpy()          # the allocating entry point
    assert np.abs(expect).max() > 0
    for call in range(2):
        out = torch.full(expect.shape, float("nan"), device=cuda)
        job = ktm.Job(image=out, **kw)
        rc = L.ktmMigratePackedNoAlloc(C.byref(job.job))
        assert rc == 0, ktm._lib.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.isfinite(got).all(), f"call {call}"
        # same kernel, different trace-slice count: only the summation order differs
        assert _rel_l2(got, expect) < 2e-5, f"call {call}"


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
