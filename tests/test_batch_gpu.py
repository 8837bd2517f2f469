"""Batched target-oriented migration (one persistent launch) and tile tuning.

Every job's image from ktmMigrateBatch must match ktmMigrate on the same job
(the batch adds trace slices with atomics, so sums agree to FP32 rounding), for
uneven jobs: patch sizes, Nz, trace counts and velocity laws differ per job.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(dev)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def make_jobs(dev, n=6, seed=0, fmt="bf16", prefold=False):
    import ktm
    from ktm import synth
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(n):
        side = int(rng.integers(3, 17))
        ntr = int(rng.integers(200, 3000))
        sv = synth.areal_survey(ntr=ntr, side=1000.0, maxoff=800.0, nx=side, ny=side, dxy=40.0,
                                nt=300, dt=0.004, nz=int(rng.integers(150, 300)), nscat=5,
                                aperture=700.0, seed=100 + j)
        tr = synth.synthesize(sv)
        packed = ktm.prepare(_t(tr, dev), sv.dt, fmt=fmt, prefold=prefold)
        import torch
        jobs.append(dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt,
                         midX=_t(sv.midX, dev), midY=_t(sv.midY, dev), offX=_t(sv.offX, dev),
                         offY=_t(sv.offY, dev), traces=packed, velocity=_t(sv.velocity, dev),
                         pick="linear", aperture=sv.aperture,
                         image=torch.full(sv.shape, float("nan"), device=dev)))
    return jobs


@pytest.mark.parametrize("fmt,prefold", [("bf16", False), ("f16", True), ("f32", False)])
def test_batch_matches_single_jobs(cuda, ktm_lib, fmt, prefold):
    import ktm
    jobs = make_jobs(cuda, fmt=fmt, prefold=prefold)
    images = ktm.migrate_batch(jobs)
    for kw, img in zip(jobs, images):
        single = ktm.migrate(**{**kw, "image": None}).cpu().numpy()
        got = img.cpu().numpy()
        assert np.isfinite(got).all()
        assert rel_l2(got, single) < 1e-5


def test_batch_rejects_mixed_formats(cuda, ktm_lib):
    import ktm
    a = make_jobs(cuda, n=1, fmt="bf16")
    b = make_jobs(cuda, n=1, fmt="f16", seed=1)
    with pytest.raises(ktm.KtmError):
        ktm.migrate_batch(a + b)


def test_autotune_returns_a_run_and_is_remembered(cuda, ktm_lib):
    import ktm
    kw = make_jobs(cuda, n=1)[0]
    r1 = ktm.autotune(**kw)
    assert r1 in (256, 384, 512)
    assert ktm.autotune(**kw) == r1
    img = ktm.migrate(**{**kw, "image": None, "tile_run": r1}).cpu().numpy()
    ref = ktm.migrate(**{**kw, "image": None, "tile_run": 256}).cpu().numpy()
    assert rel_l2(img, ref) < 1e-5
