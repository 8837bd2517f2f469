"""Multi-GPU sharding logic on CPU ranks (gloo, world size 2 and 4).

The migration is the FP64 oracle here, so the partitioning, the FP64 trace
selection and the collectives are checked without a GPU:

* output-tile sharding: every rank images its tile with only the traces its
  aperture-grown bounding box selects; the gathered image equals the full
  single-process image bit for bit (culled traces contribute exact zeros);
* trace sharding: every rank images the whole grid from its share of the
  traces; one all_reduce / reduce sums them to the full image (FP64 sums in
  another order: equal to 1e-12);
* a rank that raises before the collective makes the others fail with an
  error (a short process-group timeout), not hang.
"""
from __future__ import annotations

import datetime
import os
import socket

import numpy as np
import pytest

import oracle
from ktm import shard


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case(seed=5, ntr=90, nt=120, nx=7, ny=5, nz=40, dt=0.004):
    rng = np.random.default_rng(seed)
    gx, gy, gz = oracle.grid(nx, 25.0, 12.5), oracle.grid(ny, 50.0, -100.0), oracle.grid(nz, 0.004, 0.0)
    mid = np.stack([rng.uniform(-300, 500, ntr), rng.uniform(-400, 300, ntr)], 1).astype(np.float32)
    off = rng.uniform(-200, 200, (ntr, 2)).astype(np.float32)
    tr = rng.standard_normal((ntr, nt)).astype(np.float32)
    vel = rng.uniform(1500, 3000, (nx, ny, nz)).astype(np.float32)
    return dict(imageX=gx, imageY=gy, imageZ=gz, dt=dt, midX=mid[:, 0].copy(), midY=mid[:, 1].copy(),
                offX=off[:, 0].copy(), offY=off[:, 1].copy(), traces=tr, velocity=vel,
                aperture=260.0)


def _oracle_migrate(*, imageX, imageY, imageZ, dt, midX, midY, offX, offY, traces, velocity,
                    aperture, **_):
    return oracle.migrate_f64(imageX, imageY, imageZ, dt, midX, midY, offX, offY, traces,
                              velocity, pick=1, aperture=aperture)


def _worker(rank, world, port, mode, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    try:
        c = _case()
        nz = c["imageZ"].imagePnts
        if mode == "tiles":
            tiles = shard.tile_partition(c["imageX"].imagePnts, c["imageY"].imagePnts, world)
            img = shard.migrate_tile(tiles[rank], migrate=_oracle_migrate, **c)
            full = shard.gather_tiles(img, tiles, nz, dst=0)
            if rank == 0:
                np.save(os.path.join(outdir, "out.npy"), full.numpy())
        elif mode in ("allreduce", "reduce"):
            dst = None if mode == "allreduce" else world - 1
            img = shard.migrate_trace_shard(migrate=_oracle_migrate, dst=dst, **c)
            if img is not None:
                np.save(os.path.join(outdir, f"out{rank}.npy"), img.numpy())
        elif mode == "fail":
            if rank == 1:
                raise RuntimeError("rank 1 fails before the collective")
            import torch
            t = torch.zeros(4)
            try:
                dist.all_reduce(t)
                np.save(os.path.join(outdir, f"noerror{rank}.npy"), t.numpy())
            except Exception:  # noqa: BLE001 -- the expected timeout / peer error
                np.save(os.path.join(outdir, f"error{rank}.npy"), np.zeros(1))
    finally:
        if mode != "fail" or rank != 1:
            try:
                dist.destroy_process_group()
            except Exception:  # noqa: BLE001
                pass


def _spawn(world, mode, tmp_path, expect_ok=True):
    import torch.multiprocessing as mp
    ctx = mp.start_processes(_worker, args=(world, _free_port(), mode, str(tmp_path)),
                             nprocs=world, join=False, start_method="spawn")
    try:
        while not ctx.join(timeout=120):
            pass
    except Exception:  # noqa: BLE001
        if expect_ok:
            raise


@pytest.mark.parametrize("nx,ny,world", [(7, 5, 2), (7, 5, 4), (200, 200, 8), (3, 1, 3), (1, 9, 4)])
def test_tile_partition_covers_grid_once(nx, ny, world):
    tiles = shard.tile_partition(nx, ny, world)
    assert len(tiles) == world
    cover = np.zeros((nx, ny), int)
    for t in tiles:
        cover[t.ix0:t.ix1, t.iy0:t.iy1] += 1
    assert (cover == 1).all()
    sizes = [t.shape[0] * t.shape[1] for t in tiles]
    assert max(sizes) - min(sizes) <= max(nx, ny)


def test_select_traces_keeps_every_contributing_trace():
    c = _case()
    tiles = shard.tile_partition(7, 5, 4)
    full = _oracle_migrate(**c)
    for t in tiles:
        idx = shard.select_traces(c["midX"], c["midY"], t, c["imageX"], c["imageY"], c["aperture"])
        assert 0 < len(idx) < len(c["midX"])
        sub = dict(c, midX=c["midX"][idx], midY=c["midY"][idx], offX=c["offX"][idx],
                   offY=c["offY"][idx], traces=c["traces"][idx])
        img = _oracle_migrate(**sub)[t.ix0:t.ix1, t.iy0:t.iy1]
        assert np.array_equal(img, full[t.ix0:t.ix1, t.iy0:t.iy1])


@pytest.mark.parametrize("world", [2, 4])
def test_output_tile_sharding_gloo(tmp_path, world):
    _spawn(world, "tiles", tmp_path)
    got = np.load(tmp_path / "out.npy")
    ref = _oracle_migrate(**_case())
    # FP32 image gathered from FP64 tiles: equal to the FP32 rounding of the full image
    assert np.array_equal(got, ref.astype(np.float32))


@pytest.mark.parametrize("mode", ["allreduce", "reduce"])
def test_trace_sharding_gloo(tmp_path, mode):
    _spawn(2, mode, tmp_path)
    ref = _oracle_migrate(**_case())
    outs = sorted(tmp_path.glob("out*.npy"))
    assert len(outs) == (2 if mode == "allreduce" else 1)
    for o in outs:
        got = np.load(o)
        assert np.allclose(got, ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())


def test_failed_rank_makes_peers_error_not_hang(tmp_path):
    _spawn(2, "fail", tmp_path, expect_ok=False)
    assert (tmp_path / "error0.npy").exists()
    assert not (tmp_path / "noerror0.npy").exists()
