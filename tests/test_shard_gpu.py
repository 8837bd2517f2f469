"""Output-tile sharding with the CUDA kernel, one tile after another on one GPU.

Each tile is imaged from only the traces its aperture-grown bounding box
selects (FP64, on the host) with the packed trace rows gathered on the device,
exactly as a rank of ``bench.py --gpus N`` does; the assembled tiles must equal
the full-image migration up to FP32 summation order (the trace slices of the
launches differ), and the tiles must really drop traces.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("world", [2, 4, 6])
def test_tiles_assemble_the_full_image(cuda, ktm_lib, world):
    import torch

    import ktm
    from ktm import shard, synth
    sv = synth.areal_survey(ntr=6000, side=2000.0, maxoff=900.0, nx=30, ny=22, dxy=50.0,
                            nt=400, dt=0.004, nz=300, nscat=10, freq=25.0, noise=0.05,
                            aperture=500.0, vtop=1500.0, vbot=2800.0, lateral=0.05, rho_opt=3,
                            seed=41)
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x, dtype=np.float32)).to(cuda)  # noqa: E731
    co = [T(x) for x in (sv.midX, sv.midY, sv.offX, sv.offY)]
    raw = synth.synthesize_device(sv, device=cuda, coords=co)
    packed = ktm.prepare(raw, sv.dt, fmt="f16", rho=sv.rho_opt, prefold=True)
    kw = dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt, midX=co[0],
              midY=co[1], offX=co[2], offY=co[3], traces=packed, velocity=T(sv.velocity),
              aperture=sv.aperture, pick="linear", weight="prefold")
    full = ktm.migrate(**kw).cpu().numpy()
    tiles = shard.tile_partition(sv.shape[0], sv.shape[1], world)
    assert len(tiles) == world
    img = np.full(full.shape, np.nan, np.float32)
    kept = []
    for t in tiles:
        kept.append(len(shard.select_traces(sv.midX, sv.midY, t, sv.imageX, sv.imageY,
                                            sv.aperture)))
        img[t.ix0:t.ix1, t.iy0:t.iy1] = shard.migrate_tile(t, **kw).cpu().numpy()
    assert np.isfinite(img).all()
    assert min(kept) < sv.ntr            # the host cull drops traces
    assert rel_l2(img, full) < 1e-6
