"""Bad inputs injected on the host (no device fault is made).

* traces far outside the image, and traces with NaN or infinite coordinates,
  contribute nothing: the image equals the image without them, in fast mode
  (aperture or not) -- their traveltime is culled or clamped onto the zero
  guard sample;
* reference mode, a NaN sample in one trace (the sample of that trace the
  reference picks most often): the NaN reaches exactly the image samples whose
  truncated pick lands on it, as in the reference's own compiled
  psktmCPU.c (oracle/_ref, one thread; the oracle restatement where it was not
  built); every other sample stays bit-identical;
* reference mode, zero / negative / 1e30 / infinite / NaN velocities and infinite
  samples: the reference's NaN and infinite image samples, through both drop-in
  entry points.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from test_parity_gpu import random_case, rel_l2

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(dev)


@pytest.mark.parametrize("aperture", [0.0, 250.0])
def test_far_and_nonfinite_coordinates_contribute_nothing(cuda, ktm_lib, aperture):
    import ktm
    gx, gy, gz, dt, mx, my, ox, oy, tr, vel = random_case(41, ntr=200, data="band")
    bad = 6
    mxb = np.concatenate([mx, [1.0e6, -2.0e6, np.nan, 0.0, np.inf, 0.0]]).astype(np.float32)
    myb = np.concatenate([my, [0.0, 5.0e5, 0.0, np.nan, 0.0, -np.inf]]).astype(np.float32)
    oxb = np.concatenate([ox, [10.0, 10.0, 10.0, 10.0, 10.0, np.nan]]).astype(np.float32)
    oyb = np.concatenate([oy, [0.0] * bad]).astype(np.float32)
    trb = np.concatenate([tr, np.ones((bad, tr.shape[1]), np.float32)])

    def run(mx_, my_, ox_, oy_, tr_):
        p = ktm.prepare(_t(tr_, cuda), dt, fmt="f32", prefold=True)
        return ktm.migrate(imageX=gx, imageY=gy, imageZ=gz, dt=dt, midX=_t(mx_, cuda),
                           midY=_t(my_, cuda), offX=_t(ox_, cuda), offY=_t(oy_, cuda), traces=p,
                           velocity=_t(vel, cuda), pick="linear", aperture=aperture,
                           weight="prefold").cpu().numpy()

    good = run(mx, my, ox, oy, tr)
    withbad = run(mxb, myb, oxb, oyb, trb)
    assert np.isfinite(withbad).all()
    assert rel_l2(withbad, good) < 1e-6


def _most_picked_sample(gx, gy, gz, dt, mx, my, ox, oy, vel, k, nt):
    """The sample of trace k that the reference picks for the most image points,
    found on the CPU by migrating that trace alone as one spike after another."""
    best, hits = -1, 0
    for s in range(nt):
        spike = np.zeros((1, nt), np.float32)
        spike[0, s] = 1.0
        img = oracle.migrate_ref32(gx, gy, gz, dt, mx[k:k + 1], my[k:k + 1], ox[k:k + 1],
                                   oy[k:k + 1], spike, vel)
        n = int(np.count_nonzero(img))
        if n > hits:
            best, hits = s, n
    return best


def test_nan_sample_reaches_the_reference_picks(cuda, ktm_lib):
    import ktm
    gx, gy, gz, dt, mx, my, ox, oy, tr, vel = random_case(43, ntr=40, nt=120, nz=90, data="band")
    tr = tr.copy()
    s = _most_picked_sample(gx, gy, gz, dt, mx, my, ox, oy, vel, 7, tr.shape[1])
    assert s >= 0
    tr[7, s] = np.nan
    cfg = ktm.JobParams(tr.shape[0], tr.shape[1], dt)
    got = ktm.ktmMigrationGPU(gx, gy, gz, cfg, mx, my, ox, oy, tr, vel)
    if oracle.ref_available():
        ref = oracle.migrate_reference_c(gx, gy, gz, dt, mx, my, ox, oy, tr, vel, threads=1)
    else:
        ref = oracle.migrate_ref32(gx, gy, gz, dt, mx, my, ox, oy, tr, vel)
    assert 0 < np.isnan(ref).sum() < ref.size           # picked somewhere, not everywhere
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    fin = ~np.isnan(ref)
    assert np.array_equal(got[fin].view(np.uint32), ref[fin].view(np.uint32))


@pytest.mark.parametrize("entry", ["ktmMigrationCPU", "ktmMigrationGPU"])
def test_degenerate_velocity_and_samples_reference_mode(cuda, ktm_lib, entry):
    """Zero, negative, 1e30, infinite and NaN velocities and infinite trace samples
    through the drop-in entry points: the same NaN and infinite image samples as the
    reference's own compiled psktmCPU.c (one thread; the oracle restatement where it
    was not built), every other sample bit-identical."""
    import ktm
    from conftest import degenerate_reference_case, same_with_nans
    gx, gy, gz, dt, mx, my, ox, oy, tr, vel = degenerate_reference_case()
    cfg = ktm.JobParams(tr.shape[0], tr.shape[1], dt)
    got = getattr(ktm, entry)(gx, gy, gz, cfg, mx, my, ox, oy, tr, vel)
    if oracle.ref_available():
        ref = oracle.migrate_reference_c(gx, gy, gz, dt, mx, my, ox, oy, tr, vel, threads=1)
    else:
        ref = oracle.migrate_ref32(gx, gy, gz, dt, mx, my, ox, oy, tr, vel)
    assert np.isnan(ref).any() and np.isinf(ref).any()
    assert same_with_nans(got, ref)
