"""Seeded synthetic traces on the device (ktmSynthesizeTraces): the benchmark's
input.  Two runs give the same bits (each sample sums the scatterers in order),
and the traces agree with the numpy recipe of ktm/synth.py (FP64 sums) to FP32
rounding of the per-sample sums."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("noise", [0.0, 0.05])
def test_device_synthesis_repeatable_and_matches_numpy(cuda, ktm_lib, noise):
    import torch

    from ktm import synth
    sv = synth.areal_survey(ntr=3000, side=2000.0, maxoff=900.0, nx=8, ny=8, dxy=50.0, nt=700,
                            dt=0.002, nz=300, nscat=60, freq=30.0, noise=noise, aperture=500.0,
                            vtop=1500.0, vbot=2800.0, lateral=0.05, rho_opt=3, seed=17)
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x, dtype=np.float32)).to(cuda)  # noqa: E731
    co = [T(x) for x in (sv.midX, sv.midY, sv.offX, sv.offY)]
    a = synth.synthesize_device(sv, device=cuda, coords=co).cpu().numpy()
    b = synth.synthesize_device(sv, device=cuda, coords=co).cpu().numpy()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    # the C ABI takes the sample interval as a float (as the reference's jobParams
    # does): the numpy recipe runs with the same float-rounded interval
    ref = synth.synthesize(dataclasses.replace(sv, dt=float(np.float32(sv.dt))), noise=noise > 0)
    assert np.abs(ref).max() > 0
    err = np.linalg.norm(a.astype(np.float64) - ref) / np.linalg.norm(ref)
    assert err < 1e-6, err
