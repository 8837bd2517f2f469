"""Demigration (the adjoint), the Vrms gradient and least-squares migration.

* demigration against the FP64 oracle's transpose (same formulation), also with
  6000-sample traces and a coarse tau step;
* dot-product tests <L m, d> = <m, L^T d> to 1e-5 (seeded Gaussian m and d),
  including the 512 CMP x 64 offset x 1001 sample line of the adjoint/LSM
  configuration;
* the Vrms gradient against the FP64 oracle gradient and against central
  finite differences (eps = 1e-3 v);
* CGLS: monotone residual, graph replay equal to plain launches, and the
  torch.autograd wrappers.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)).to(dev)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def line_op(dev, ncmp=48, noff=8, nt=300, nz=260, aperture=0.0, pick="linear", weight="table",
            seed=3, dtau=None):
    from ktm import synth
    from ktm.inverse import MigrationOperator
    sv = synth.line_survey(ncmp=ncmp, noff=noff, doff=100.0, nt=nt, nz=nz, seed=seed, dtau=dtau)
    op = MigrationOperator(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt, nt=nt,
                           midX=_t(sv.midX, dev), midY=_t(sv.midY, dev), offX=_t(sv.offX, dev),
                           offY=_t(sv.offY, dev), velocity=_t(sv.velocity, dev),
                           aperture=aperture, pick=pick, weight=weight)
    return sv, op


@pytest.mark.parametrize("pick,weight", [("linear", "table"), ("truncate", "table"),
                                         ("linear", "prefold")])
def test_demigrate_matches_oracle_transpose(cuda, ktm_lib, pick, weight):
    # truncation: a tau step incommensurate with dt (see test_parity_gpu.py)
    sv, op = line_op(cuda, aperture=400.0, pick=pick, weight=weight,
                     dtau=0.00173 if pick == "truncate" else None)
    m = np.random.default_rng(1).standard_normal(op.shape).astype(np.float32)
    d = op.demigrate(_t(m, cuda)).cpu().numpy()
    ref = oracle.demigrate_f64(sv.imageX, sv.imageY, sv.imageZ, sv.dt, sv.midX, sv.midY, sv.offX,
                               sv.offY, sv.nt, sv.velocity, m, pick=1 if pick == "linear" else 0,
                               aperture=400.0, prefold=1 if weight == "prefold" else 3)
    assert not d[:, 0].any() and not d[:, sv.nt:].any()           # guards stay zero
    # each data sample sums many FP32 contributions (5e-5); truncation: index flips
    # at FP32 rounding of t/dt move a white-noise model's contributions one sample
    tol = 5e-5 if pick == "linear" else 1e-2
    assert rel_l2(d[:, :sv.nt], ref) < tol


@pytest.mark.parametrize("weight", ["table", "prefold"])
def test_demigrate_long_traces_coarse_tau(cuda, ktm_lib, weight):
    """6000-sample traces (padded accumulator rows of ~30 KB: a few traces per chunk)
    and a tau step of 1.25 dt, so t/dt moves on by two or more samples between a lane's
    consecutive tau samples (the merge flushes both samples of its pick) -- against the
    FP64 oracle's transpose."""
    sv, op = line_op(cuda, ncmp=16, noff=4, nt=6000, nz=300, aperture=400.0, weight=weight,
                     dtau=0.005)
    m = np.random.default_rng(2).standard_normal(op.shape).astype(np.float32)
    d = op.demigrate(_t(m, cuda)).cpu().numpy()
    ref = oracle.demigrate_f64(sv.imageX, sv.imageY, sv.imageZ, sv.dt, sv.midX, sv.midY, sv.offX,
                               sv.offY, sv.nt, sv.velocity, m, pick=1, aperture=400.0,
                               prefold=1 if weight == "prefold" else 3)
    assert np.abs(ref).max() > 0
    assert not d[:, 0].any() and not d[:, sv.nt:].any()
    # t/dt reaches ~750 samples here, where the FP32 square roots move f by ~1e-4 of a
    # sample, and each data sample sums fewer contributions than on the finer tau grid
    assert rel_l2(d[:, :sv.nt], ref) < 1e-4


@pytest.mark.parametrize("pick,weight,aperture", [("linear", "table", 0.0), ("linear", "table", 300.0),
                                                  ("linear", "sqrt", 0.0), ("truncate", "table", 0.0),
                                                  ("linear", "prefold", 0.0),
                                                  ("linear", "prefold", 300.0)])
def test_dot_product(cuda, ktm_lib, pick, weight, aperture):
    import torch
    sv, op = line_op(cuda, aperture=aperture, pick=pick, weight=weight)
    rng = np.random.default_rng(7)
    m = _t(rng.standard_normal(op.shape), cuda)
    d = op.pack(_t(rng.standard_normal((op.ntr, sv.nt)), cuda))
    Lm = op.demigrate(m)
    Ltd = op.migrate(d)
    lhs = torch.dot(Lm.double().flatten(), d.double().flatten()).item()
    rhs = torch.dot(m.double().flatten(), Ltd.double().flatten()).item()
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


@pytest.mark.parametrize("weight", ["table", "prefold"])
def test_dot_product_adjoint_config(cuda, ktm_lib, weight):
    """512 CMPs x 64 offsets x 1001 samples at 4 ms, seeded Gaussian model and data."""
    import torch
    sv, op = line_op(cuda, ncmp=512, noff=64, nt=1001, nz=1001, seed=4, weight=weight)
    rng = np.random.default_rng(11)
    m = _t(rng.standard_normal(op.shape), cuda)
    d = op.pack(_t(rng.standard_normal((op.ntr, sv.nt)), cuda))
    lhs = torch.dot(op.demigrate(m).double().flatten(), d.double().flatten()).item()
    rhs = torch.dot(m.double().flatten(), op.migrate(d).double().flatten()).item()
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def _ricker_line(cuda, seed=5):
    import ktm
    from ktm import synth
    sv, op = line_op(cuda, ncmp=40, noff=6, nt=400, nz=300, seed=seed)
    tr = synth.synthesize(sv, noise=False)
    packed = ktm.prepare(_t(tr, cuda), sv.dt, fmt="f32", prefold=False)
    return sv, op, tr, packed


def test_vrms_gradient_matches_oracle(cuda, ktm_lib):
    sv, op, tr, packed = _ricker_line(cuda)
    g = op.vrms_gradient(packed).cpu().numpy()
    ref = oracle.vrms_grad_f64(sv.imageX, sv.imageY, sv.imageZ, sv.dt, sv.midX, sv.midY, sv.offX,
                               sv.offY, tr, sv.velocity, prefold=3)
    ref[:, :, 0] = 0.0
    assert np.abs(ref).max() > 0
    assert rel_l2(g, ref) < 1e-3


def test_vrms_gradient_central_differences(cuda, ktm_lib):
    """(I(v (1+eps)) - I(v (1-eps))) / (2 eps v) against dI/dv, eps = 1e-3, both in
    FP64 (oracle) and on the device.  Linear interpolation has slope jumps at the
    samples, which a finite difference straddles; on band-limited data the two
    agree to a few 1e-2 in relative L2."""
    import ktm
    sv, op, tr, packed = _ricker_line(cuda)
    eps = 1e-3
    args = (sv.imageX, sv.imageY, sv.imageZ, sv.dt, sv.midX, sv.midY, sv.offX, sv.offY, tr)
    cube = np.broadcast_to(sv.velocity, op.shape).astype(np.float32)
    ip = oracle.migrate_f64(*args, (cube * (1 + eps)).astype(np.float32), pick=1, prefold=3)
    im = oracle.migrate_f64(*args, (cube * (1 - eps)).astype(np.float32), pick=1, prefold=3)
    fd = (ip - im) / (2 * eps * cube)
    g64 = oracle.vrms_grad_f64(*args, sv.velocity, prefold=3)
    assert rel_l2(g64, fd) < 5e-2
    # device: finite differences of the device image with a velocity cube
    from ktm.inverse import MigrationOperator
    kw = dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt, nt=sv.nt,
              midX=op.midX, midY=op.midY, offX=op.offX, offY=op.offY)
    opp = MigrationOperator(velocity=_t(cube * (1 + eps), cuda), **kw)
    opm = MigrationOperator(velocity=_t(cube * (1 - eps), cuda), **kw)
    fd_dev = ((opp.migrate(packed.data) - opm.migrate(packed.data)).cpu().numpy() /
              (2 * eps * cube))
    g = op.vrms_gradient(packed).cpu().numpy()
    assert rel_l2(g, fd_dev) < 5e-2
    assert ktm is not None


@pytest.mark.parametrize("use_graph,weight", [(True, "table"), (False, "table"), (True, "prefold")])
def test_least_squares_migration(cuda, ktm_lib, use_graph, weight):
    import torch
    sv, op = line_op(cuda, ncmp=128, noff=16, nt=501, nz=501, seed=9, weight=weight)
    rng = np.random.default_rng(2)
    m_true = np.where(rng.uniform(size=op.shape) < 0.05, rng.standard_normal(op.shape), 0.0)
    d = op.demigrate(_t(m_true, cuda))
    model, rn, gn = op.least_squares(d, 20, use_graph=use_graph)
    print("residual norms", rn / rn[0], "gradient norms", gn / gn[0])
    assert np.all(np.diff(rn) <= 1e-6 * rn[0])            # CGLS: ||r|| never increases
    assert rn[-1] < 0.8 * rn[0]
    assert gn[-1] < 0.5 * gn[0]
    # the data misfit of the returned model matches the last recorded norm
    r = d - op.demigrate(model)
    assert abs(torch.linalg.norm(r.double()).item() - rn[-1]) <= 1e-3 * rn[0]


def test_least_squares_graph_equals_launches(cuda, ktm_lib):
    sv, op = line_op(cuda, ncmp=64, noff=8, nt=300, nz=300, seed=12)
    rng = np.random.default_rng(3)
    m_true = np.where(rng.uniform(size=op.shape) < 0.05, rng.standard_normal(op.shape), 0.0)
    d = op.demigrate(_t(m_true, cuda))
    a, rna, _ = op.least_squares(d, 8, use_graph=True)
    b, rnb, _ = op.least_squares(d, 8, use_graph=False)
    # the same launch sequence; demigration sums with shared-memory atomics, whose
    # order differs run to run at FP32 rounding, and CG carries that forward
    assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-3
    assert np.allclose(rna, rnb, rtol=1e-3)


def test_autograd_wrappers(cuda, ktm_lib):
    import torch
    from ktm.inverse import demigrate_fn
    sv, op = line_op(cuda)
    Demigrate = demigrate_fn()
    rng = np.random.default_rng(4)
    m = _t(rng.standard_normal(op.shape), cuda).requires_grad_(True)
    d_obs = op.pack(_t(rng.standard_normal((op.ntr, sv.nt)), cuda))
    loss = 0.5 * ((Demigrate.apply(m, op) - d_obs) ** 2).sum()
    loss.backward()
    expect = op.migrate(op.demigrate(m.detach()) - d_obs)
    # demigration accumulates with shared-memory atomics: sums agree to FP32 rounding
    assert rel_l2(m.grad.cpu().numpy(), expect.cpu().numpy()) < 1e-5


def test_trace_sharded_cgls_on_one_rank_matches_library(cuda, ktm_lib):
    """ktm.shard.least_squares_trace_shard (the CGLS that shards traces over
    ranks; here one rank, no process group) with the CUDA operator pair takes
    the same steps as ktmLeastSquaresMigrate."""
    import torch
    from ktm import shard
    sv, op = line_op(cuda, ncmp=64, noff=8, nt=300, nz=300, seed=12, weight="prefold")
    rng = np.random.default_rng(3)
    m_true = np.where(rng.uniform(size=op.shape) < 0.05, rng.standard_normal(op.shape), 0.0)
    d = op.demigrate(_t(m_true, cuda))
    a, rna, gna = op.least_squares(d, 8, use_graph=True)
    b, rnb, gnb = shard.least_squares_trace_shard(op.migrate, op.demigrate, d.clone(),
                                                  torch.zeros(op.shape, device=cuda), 8)
    assert np.allclose(rna, rnb, rtol=1e-3) and np.allclose(gna, gnb, rtol=1e-3)
    assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-3
