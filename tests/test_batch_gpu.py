"""Batched target-oriented migration (one persistent launch) and tile tuning.

Every job's image from ktmMigrateBatch must match ktmMigrate on the same job
(the batch adds trace slices with atomics, so sums agree to FP32 rounding), for
uneven jobs: patch sizes, Nz, trace counts and velocity laws differ per job;
and every job of a batch in the benchmark's format (FP16 with a per-trace
scale, sqrt(j dt) folded in, the rho filter on the device) must be within 1e-3
relative L2 of the CPU FP64 oracle of the whole pipeline (oracle/rho.py, then
oracle.migrate_f64 with the reference weight |tau| sqrt(t) per pair).
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


def _tune_job(cuda, ntr=3000, side=20, nz=300, nt=350, fmt="f16", seed=90):
    """One band-limited areal job (2.5-D rho on the device, sqrt(j dt) folded in) and
    its FP64 oracle image."""
    import ktm
    from ktm import synth
    sv = synth.areal_survey(ntr=ntr, side=side * 25.0 + 1200.0, maxoff=900.0, nx=side, ny=side,
                            dxy=25.0, nt=nt, dt=0.004, nz=nz, nscat=8, freq=25.0, noise=0.05,
                            aperture=600.0, vtop=1500.0, vbot=2600.0, lateral=0.0, rho_opt=2,
                            seed=seed)
    sv.imageX.imageStart = sv.imageY.imageStart = 600.0
    raw = synth.synthesize(sv)
    packed = ktm.prepare(_t(raw, cuda), sv.dt, fmt=fmt, rho=sv.rho_opt, prefold=True)
    kw = dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt,
              midX=_t(sv.midX, cuda), midY=_t(sv.midY, cuda), offX=_t(sv.offX, cuda),
              offY=_t(sv.offY, cuda), traces=packed, velocity=_t(sv.velocity, cuda),
              pick="linear", aperture=sv.aperture, weight="prefold")
    return sv, raw, kw


def test_every_tile_candidate_matches_the_oracle(cuda, ktm_lib):
    """Every shape the tuner may choose (tau run x columns per CTA x chunk) gives the
    default shape's image up to FP32 summation order, and the FP64 oracle's to 1e-3."""
    import ktm
    sv, raw, kw = _tune_job(cuda)
    ref = _oracle_pipeline(sv, raw)
    base = ktm.migrate(**kw).cpu().numpy()
    cands = ktm.tile_candidates(**kw)
    assert len(cands) == 18
    assert {c["tileCols"] for c in cands} == {24, 12, 8}
    for c in cands:
        img = ktm.migrate(tile=c, **kw).cpu().numpy()
        assert np.isfinite(img).all(), c
        assert rel_l2(img, base) < 1e-5, c
        assert rel_l2(img, ref) < 1e-3, c
    # paths built for the default shape only: truncating pick, sqrt weight
    tkw = dict(kw, traces=ktm.prepare(_t(raw, cuda), sv.dt, fmt="f16", prefold=False),
               pick="truncate", weight="sqrt")
    assert {c["tileCols"] for c in ktm.tile_candidates(**tkw)} == {24}
    with pytest.raises(ktm.KtmError):
        ktm.migrate(tile_cols=8, **tkw)


def test_autotune_tile_is_within_5_percent_of_the_best(cuda, ktm_lib):
    """The tuner's choice against an exhaustive re-timing of all its candidates on the
    same job (median of five launches each); remembered per job shape."""
    import torch

    import ktm
    _, _, kw = _tune_job(cuda, ntr=4096, side=48, nz=751, nt=751, seed=91)
    kw["image"] = torch.empty((48, 48, 751), device=cuda)
    best = ktm.autotune_tile(**kw)
    assert best["tileRun"] in (256, 384, 512) and best["tileCols"] in (24, 12, 8)
    assert best["ms"] > 0
    assert ktm.autotune_tile(**kw) == best

    def timed(tile, reps=5):
        for _ in range(2):
            ktm.migrate(tile=tile, **kw)
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            ktm.migrate(tile=tile, **kw)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    sweep = {tuple(sorted(c.items())): timed(c) for c in ktm.tile_candidates(**kw)}
    fastest = min(sweep.values())
    assert timed(best, reps=9) <= 1.05 * fastest, (best, fastest)


def test_batch_takes_a_tuned_tile(cuda, ktm_lib):
    """The batched launch runs the tuned shape; images equal the default shape's."""
    import ktm
    jobs = make_jobs(cuda, fmt="f16", prefold=True)
    for kw in jobs:
        kw["weight"] = "prefold"
    base = [img.clone() for img in ktm.migrate_batch(jobs)]
    for cols in (12, 8):
        for kw in jobs:
            kw["tile"] = {"tileRun": 384, "tileCols": cols, "tileChunk": 0}
        for img, b in zip(ktm.migrate_batch(jobs), base):
            assert rel_l2(img.cpu().numpy(), b.cpu().numpy()) < 1e-5


def _oracle_pipeline(sv, raw):
    """FP64 rho filter (ktmApplyRhoFilter.m) and FP64 migration of one job, on the CPU."""
    import oracle
    import rho
    filt = rho.rho_filter_traces(raw, sv.dt * 1e6, sv.rho_opt)
    return oracle.migrate_f64(sv.imageX, sv.imageY, sv.imageZ, sv.dt, sv.midX, sv.midY, sv.offX,
                              sv.offY, filt.astype(np.float32), sv.velocity, pick=1,
                              aperture=sv.aperture)


@pytest.mark.parametrize("fmt,gate", [("f16", 1e-3), ("bf16", 4e-3)])
def test_batch_jobs_against_fp64_oracle(cuda, ktm_lib, fmt, gate):
    """Per-job error of the batched launch against the FP64 oracle.  FP16 (the
    batch benchmark's format) is held to the 1e-3 bar on every job.  BF16 keeps 8
    significant bits (relative rounding error up to 2^-9 per sample), and these
    patches sum too few coherent traces for it to average out: it measures
    1.1e-3 to 1.4e-3 on them, so it is held to 4e-3 here; the 1e-3 claim for BF16
    holds on the full 2-D line (tests/test_full_size_gpu.py)."""
    import torch

    import ktm
    from ktm import synth
    rng = np.random.default_rng(77)
    jobs, refs = [], []
    for j in range(5):
        side = int(rng.integers(4, 14))
        ntr = int(rng.integers(800, 2500))
        sv = synth.areal_survey(ntr=ntr, side=side * 25.0 + 1200.0, maxoff=900.0, nx=side,
                                ny=side, dxy=25.0, nt=350, dt=0.004, nz=int(rng.integers(200, 350)),
                                nscat=8, freq=25.0, noise=0.05, aperture=600.0, vtop=1500.0,
                                vbot=2600.0, lateral=0.0, rho_opt=2, seed=300 + j)
        sv.imageX.imageStart = sv.imageY.imageStart = 600.0
        raw = synth.synthesize(sv)
        refs.append(_oracle_pipeline(sv, raw))
        packed = ktm.prepare(_t(raw, cuda), sv.dt, fmt=fmt, rho=sv.rho_opt, prefold=True)
        jobs.append(dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt,
                         midX=_t(sv.midX, cuda), midY=_t(sv.midY, cuda), offX=_t(sv.offX, cuda),
                         offY=_t(sv.offY, cuda), traces=packed, velocity=_t(sv.velocity, cuda),
                         pick="linear", aperture=sv.aperture,
                         image=torch.full(sv.shape, float("nan"), device=cuda)))
    images = ktm.migrate_batch(jobs)
    errs = [rel_l2(img.cpu().numpy(), ref) for img, ref in zip(images, refs)]
    assert all(np.abs(r).max() > 0 for r in refs)
    assert max(errs) < gate, errs


def test_batch_edge_jobs(cuda, ktm_lib):
    """Jobs with no traces (image overwritten with zeros), a 1 x 1 image, a single trace,
    and the tuner on a job with nothing to time (the default tile)."""
    import torch

    import ktm
    jobs = make_jobs(cuda, n=3, fmt="f16", prefold=True, seed=5)
    for kw in jobs:
        kw["weight"] = "prefold"
    empty = dict(jobs[0])
    empty["traces"] = ktm.api.PackedTraces(jobs[0]["traces"].data[:0], jobs[0]["traces"].scale[:0],
                                           jobs[0]["traces"].nt, "f16", True, 0)
    for k in ("midX", "midY", "offX", "offY"):
        empty[k] = jobs[0][k][:0]
    empty["image"] = torch.full(jobs[0]["image"].shape, float("nan"), device=cuda)
    one = dict(jobs[1])
    one["imageX"] = ktm.grid(1, one["imageX"].imageStep, one["imageX"].imageStart)
    one["imageY"] = ktm.grid(1, one["imageY"].imageStep, one["imageY"].imageStart)
    one["velocity"] = one["velocity"][:1, :1].contiguous()
    one["image"] = torch.full((1, 1, jobs[1]["imageZ"].imagePnts), float("nan"), device=cuda)
    single = dict(jobs[2])
    single["traces"] = ktm.api.PackedTraces(jobs[2]["traces"].data[:1], jobs[2]["traces"].scale[:1],
                                            jobs[2]["traces"].nt, "f16", True, 0)
    for k in ("midX", "midY", "offX", "offY"):
        single[k] = jobs[2][k][:1]
    single["image"] = torch.full(jobs[2]["image"].shape, float("nan"), device=cuda)
    imgs = ktm.migrate_batch([empty, one, single])
    assert torch.count_nonzero(imgs[0]).item() == 0 and torch.isfinite(imgs[0]).all()
    for kw, img in zip([one, single], imgs[1:]):
        ref = ktm.migrate(**{**kw, "image": None}).cpu().numpy()
        assert np.isfinite(img.cpu().numpy()).all()
        assert rel_l2(img.cpu().numpy(), ref) < 1e-5 or np.abs(ref).max() == 0
    tile = ktm.autotune_tile(**empty)      # nothing to time: a valid tile, no launch
    assert tile["tileCols"] in (24, 12, 8) and tile["tileRun"] in (256, 384, 512)
