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


def _lsm_ops(c, sl):
    """Oracle L_k^T / L_k for the traces in slice sl (FP64, torch tensors)."""
    import torch
    geo = (c["imageX"], c["imageY"], c["imageZ"], c["dt"], c["midX"][sl], c["midY"][sl],
           c["offX"][sl], c["offY"][sl])
    nt = c["traces"].shape[1]

    def migrate(r):
        return torch.from_numpy(oracle.migrate_f64(*geo, r.numpy().astype(np.float32), c["velocity"],
                                                   pick=1, aperture=c["aperture"]))

    def demigrate(m):
        return torch.from_numpy(oracle.demigrate_f64(*geo, nt, c["velocity"], m.numpy(), pick=1,
                                                     aperture=c["aperture"]))
    return migrate, demigrate


def _lsm_case():
    """Data demigrated (FP64, float32-representable) from a sparse seeded model."""
    import torch
    c = _case(ntr=48, nt=80, nx=5, ny=3, nz=30)
    rng = np.random.default_rng(8)
    shape = (5, 3, 30)
    m_true = np.where(rng.uniform(size=shape) < 0.1, rng.standard_normal(shape), 0.0)
    _, dem = _lsm_ops(c, slice(0, 48))
    d = dem(torch.from_numpy(m_true)).numpy().astype(np.float32).astype(np.float64)
    return c, torch.from_numpy(d), shape


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
        elif mode == "lsm":
            import torch
            c, d, shape = _lsm_case()
            sl = shard.trace_shard(d.shape[0], rank, world)
            mig, dem = _lsm_ops(c, sl)
            m, rn, gn = shard.least_squares_trace_shard(mig, dem, d[sl].clone(),
                                                        torch.zeros(shape, dtype=torch.float64), 6)
            np.savez(os.path.join(outdir, f"lsm{rank}.npz"), m=m.numpy(), rn=rn, gn=gn)
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


def test_least_squares_trace_sharding_gloo(tmp_path):
    """CGLS with the traces split over 2 ranks (one image all_reduce and two FP64
    scalar all_reduces per iteration) equals the single-process CGLS over all
    traces, every rank holding the same model."""
    import torch
    _spawn(2, "lsm", tmp_path)
    c, d, shape = _lsm_case()
    mig, dem = _lsm_ops(c, slice(0, d.shape[0]))
    m, rn, gn = shard.least_squares_trace_shard(mig, dem, d.clone(),
                                                torch.zeros(shape, dtype=torch.float64), 6)
    assert rn[-1] < 0.5 * rn[0] and np.all(np.diff(rn) <= 1e-12 * rn[0])
    for k in range(2):
        z = np.load(tmp_path / f"lsm{k}.npz")
        assert np.allclose(z["rn"], rn, rtol=1e-9) and np.allclose(z["gn"], gn, rtol=1e-9)
        assert np.allclose(z["m"], m.numpy(), rtol=1e-8, atol=1e-10 * np.abs(m.numpy()).max())


def test_least_squares_trace_shard_solves_a_dense_system():
    """The CGLS of least_squares_trace_shard on one rank with dense operators
    (L = A, L^T = A^T): it reaches the least-squares solution of an
    overdetermined system, and ||r|| never increases."""
    import torch
    rng = np.random.default_rng(21)
    A = torch.from_numpy(rng.standard_normal((60, 14)))
    b = torch.from_numpy(rng.standard_normal(60))
    x, rn, gn = shard.least_squares_trace_shard(lambda r: A.T @ r, lambda m: A @ m, b.clone(),
                                                torch.zeros(14, dtype=torch.float64), 40)
    ref = np.linalg.lstsq(A.numpy(), b.numpy(), rcond=None)[0]
    assert np.allclose(x.numpy(), ref, rtol=1e-8, atol=1e-10)
    assert np.all(np.diff(rn) <= 1e-12 * rn[0])
    assert gn[-1] < 1e-8 * gn[0]
