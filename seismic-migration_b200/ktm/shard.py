"""Multi-GPU migration, one process per GPU (torch.distributed).

Output points are independent sums over traces, so the image shards without
any exchange in the data path:

* ``tile_partition`` splits the (x, y) image grid into one rectangle per rank
  (balanced in columns);
* ``select_traces`` keeps the traces that can reach a tile: midpoints inside
  the tile's bounding box grown by the aperture, decided in FP64 on the host
  (a trace outside contributes exactly zero there, because the kernels skip
  pairs with |mid - x| > aperture);
* ``migrate_tile`` images one rank's tile with its traces; ``gather_tiles``
  assembles the full image on one rank (the only collective, optional).

For a small image with very many traces the alternative is to shard the
traces and sum the images once (``migrate_trace_shard``: one ``all_reduce``
or ``reduce`` of the FP32 image).  Least-squares migration shards the same way
(``least_squares_trace_shard``: per CGLS iteration one ``all_reduce`` of the
image and two of an FP64 scalar).

The migration itself is a callable (``ktm.migrate`` by default) so that the
partitioning and the collectives can be exercised on CPU ranks (gloo).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from ._lib import ImageGrid


@dataclass(frozen=True)
class Tile:
    """Image columns [ix0, ix1) x [iy0, iy1) of the full grid."""
    ix0: int
    ix1: int
    iy0: int
    iy1: int

    @property
    def shape(self):
        return (self.ix1 - self.ix0, self.iy1 - self.iy0)

    def grids(self, gx: ImageGrid, gy: ImageGrid):
        """Sub-grids of the tile: start' = the full axis value at ix0 (iy0),
        start + (float)ix0 * step in float as psktmFunctions.c:19-39 forms it,
        same step.  The tile's axis start' + (float)i' * step then equals the
        full axis at ix0 + i' exactly when those sums are exact in float (grid
        starts and steps with few significant bits, as survey grids have),
        and within one rounding otherwise."""
        sx = np.float32(gx.imageStart) + np.float32(self.ix0) * np.float32(gx.imageStep)
        sy = np.float32(gy.imageStart) + np.float32(self.iy0) * np.float32(gy.imageStep)
        return (ImageGrid(self.ix1 - self.ix0, float(gx.imageStep), float(sx)),
                ImageGrid(self.iy1 - self.iy0, float(gy.imageStep), float(sy)))


def _split(n: int, parts: int):
    b = [n * p // parts for p in range(parts + 1)]
    return list(zip(b[:-1], b[1:]))


def tile_partition(nx: int, ny: int, world: int) -> list[Tile]:
    """One rectangle per rank: px x py ranks with px * py = world, px chosen so
    the tiles are as square as the grid allows; every column belongs to
    exactly one tile and tile sizes differ by at most one row / column."""
    if world < 1:
        raise ValueError("world must be >= 1")
    best = None
    for px in range(1, world + 1):
        if world % px:
            continue
        py = world // px
        if px > nx or py > ny:
            continue
        # squareness of a tile, then fewer cuts along x
        cost = abs(np.log((nx / px) / max(ny / py, 1e-9)))
        if best is None or cost < best[0] - 1e-12:
            best = (cost, px, py)
    if best is None:
        raise ValueError(f"cannot split a {nx} x {ny} grid over {world} ranks")
    _, px, py = best
    return [Tile(x0, x1, y0, y1) for (x0, x1) in _split(nx, px) for (y0, y1) in _split(ny, py)]


def select_traces(midX, midY, tile: Tile, gx: ImageGrid, gy: ImageGrid, aperture: float):
    """Indices of the traces whose midpoint lies within ``aperture`` (plus a
    relative margin of 1e-6 for the float rounding of the kernels' distance)
    of the tile's bounding box, in FP64.  ``aperture <= 0`` keeps every trace."""
    mx = np.asarray(midX, np.float64)
    my = np.asarray(midY, np.float64)
    if aperture <= 0:
        return np.arange(mx.size)
    ax = lambda g, i: float(np.float32(g.imageStart) + np.float32(i) * np.float32(g.imageStep))  # noqa: E731
    xs = (ax(gx, tile.ix0), ax(gx, tile.ix1 - 1))
    ys = (ax(gy, tile.iy0), ax(gy, tile.iy1 - 1))
    x0, x1 = min(xs), max(xs)
    y0, y1 = min(ys), max(ys)
    r = float(aperture) * (1.0 + 1e-6) + 1e-3
    dx = np.maximum(np.maximum(x0 - mx, mx - x1), 0.0)
    dy = np.maximum(np.maximum(y0 - my, my - y1), 0.0)
    return np.nonzero(dx * dx + dy * dy <= r * r)[0]


def take_rows(a, idx):
    """Rows ``idx`` of a numpy array, a torch tensor (gathered on its device) or a
    packed trace set (samples and per-trace scales)."""
    from .api import PackedTraces
    if isinstance(a, PackedTraces):
        return PackedTraces(take_rows(a.data, idx), take_rows(a.scale, idx), a.nt, a.fmt,
                            a.prefolded, a.rho)
    if hasattr(a, "index_select"):
        import torch
        return a.index_select(0, torch.as_tensor(np.asarray(idx, np.int64), device=a.device))
    return a[idx]


def tile_velocity(velocity, tile: Tile):
    """A 1-D velocity as is; a [Nx, Ny, Nz] cube cut to the tile (contiguous)."""
    if len(getattr(velocity, "shape", ())) != 3:
        return velocity
    v = velocity[tile.ix0:tile.ix1, tile.iy0:tile.iy1]
    return v.contiguous() if hasattr(v, "contiguous") else np.ascontiguousarray(v)


def migrate_tile(tile: Tile, *, imageX, imageY, imageZ, midX, midY, offX, offY, traces,
                 velocity, aperture=0.0, migrate=None, take=None, **kw):
    """Image one tile with the traces that reach it.  ``velocity`` is 1-D or the
    full [Nx, Ny, Nz] cube (cut to the tile).  ``take(array, indices)`` gathers
    the selected traces (``take_rows`` by default: numpy arrays, torch tensors on
    their device, packed trace sets).  Returns the tile image [tnx, tny, Nz]."""
    if migrate is None:
        from .api import migrate as migrate   # noqa: PLW0127
    if take is None:
        take = take_rows
    mx = midX.cpu().numpy() if hasattr(midX, "cpu") else midX
    my = midY.cpu().numpy() if hasattr(midY, "cpu") else midY
    idx = select_traces(mx, my, tile, imageX, imageY, aperture)
    tgx, tgy = tile.grids(imageX, imageY)
    return migrate(imageX=tgx, imageY=tgy, imageZ=imageZ, midX=take(midX, idx),
                   midY=take(midY, idx), offX=take(offX, idx), offY=take(offY, idx),
                   traces=take(traces, idx), velocity=tile_velocity(velocity, tile),
                   aperture=aperture, **kw)


def gather_tiles(tile_image, tiles: list[Tile], nz: int, group=None, dst: int | None = 0):
    """Assemble the full [Nx, Ny, Nz] image from every rank's tile with one
    ``all_gather`` of equal-size padded buffers (gloo and NCCL both support
    it).  Returns the image on rank ``dst`` (every rank when dst is None),
    None elsewhere."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    if len(tiles) != world:
        raise ValueError("one tile per rank expected")
    t = torch.as_tensor(tile_image)
    cap = max(tt.shape[0] * tt.shape[1] for tt in tiles) * nz
    buf = torch.zeros(cap, dtype=torch.float32, device=t.device)
    flat = t.reshape(-1).to(torch.float32)
    buf[: flat.numel()] = flat
    outs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf, group=group)
    if dst is not None and rank != dst:
        return None
    nx = max(tt.ix1 for tt in tiles)
    ny = max(tt.iy1 for tt in tiles)
    full = torch.empty((nx, ny, nz), dtype=torch.float32, device=t.device)
    for tt, o in zip(tiles, outs):
        a, b = tt.shape
        full[tt.ix0:tt.ix1, tt.iy0:tt.iy1] = o[: a * b * nz].reshape(a, b, nz)
    return full


def trace_shard(ntr: int, rank: int, world: int) -> slice:
    """Contiguous, balanced share of the traces for one rank."""
    a, b = _split(ntr, world)[rank]
    return slice(a, b)


def migrate_trace_shard(*, midX, midY, offX, offY, traces, group=None, dst: int | None = None,
                        migrate=None, **kw):
    """Shard the traces, image the whole grid on every rank, then sum the
    images with one collective: ``all_reduce`` (dst None) or ``reduce`` to
    rank dst.  Returns the summed image (on every rank, or on dst)."""
    import torch
    import torch.distributed as dist
    if migrate is None:
        from .api import migrate as migrate   # noqa: PLW0127
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    s = trace_shard(len(midX), rank, world)
    img = migrate(midX=midX[s], midY=midY[s], offX=offX[s], offY=offY[s], traces=traces[s], **kw)
    t = torch.as_tensor(img)
    if dst is None:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t
    dist.reduce(t, dst=dst, op=dist.ReduceOp.SUM, group=group)
    return t if rank == dst else None


def least_squares_trace_shard(migrate, demigrate, data, model, iterations: int, group=None):
    """Least-squares migration (CGLS, as ktmLeastSquaresMigrate) with the traces
    sharded over the ranks of ``group``: rank k holds its data shard d_k and
    L = [L_0; L_1; ...] stacks the ranks' demigrations, so

        L p   = (L_k p) on each rank, no exchange;
        L^T r = sum_k L_k^T r_k: one all_reduce of the image;
        <q, q>, <r, r> = sums over ranks: all_reduce of one FP64 scalar each.

    ``migrate(r_k)`` returns L_k^T r_k (an image tensor), ``demigrate(p)`` returns
    L_k p (a data tensor shaped like ``data``).  ``model`` is the starting model,
    the same on every rank; it is updated in place and returned with the residual
    norms ||d - L m_i|| and gradient norms ||L^T (d - L m_i)|| (float64 arrays of
    iterations + 1).  Every rank takes the same collectives in the same order;
    without an initialised process group the ranks are one (no collective).
    Vectors keep the dtype and device of ``data`` / ``model``; dot products are
    FP64."""
    import torch
    import torch.distributed as dist
    sharded = dist.is_available() and dist.is_initialized()

    def allsum(t):
        if sharded:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t

    def dot(x, y):
        return torch.dot(x.reshape(-1).double(), y.reshape(-1).double())

    def scalar_sum(x):
        return float(allsum(x.reshape(1).clone())[0])

    r = data - demigrate(model)
    s = allsum(migrate(r))
    p = s.clone()
    gamma = float(dot(s, s))
    rn = np.zeros(iterations + 1)
    gn = np.zeros(iterations + 1)
    rn[0] = np.sqrt(scalar_sum(dot(r, r)))
    gn[0] = np.sqrt(gamma)
    for it in range(1, iterations + 1):
        q = demigrate(p)
        delta = scalar_sum(dot(q, q))
        alpha = gamma / delta if delta > 0.0 else 0.0
        model += alpha * p
        r -= alpha * q
        s = allsum(migrate(r))
        gamma_new = float(dot(s, s))
        beta = gamma_new / gamma if gamma > 0.0 else 0.0
        gamma = gamma_new
        p = s + beta * p
        rn[it] = np.sqrt(scalar_sum(dot(r, r)))
        gn[it] = np.sqrt(gamma)
    return model, rn, gn
