"""Known-answer tests of the method itself (analytic, no reference needed).

* single spike -> isochron: one zero-offset trace with one non-zero sample j0
  images onto the set of (x, tau) whose two-way time 2 sqrt(tau^2 + d^2/v^2)
  truncates to j0 (psktmCPU.c:80-85), an ellipse in (x, tau), with the
  reference weight |tau| sqrt(t) as amplitude;
* point diffractor -> focus: traces synthesised with a Ricker wavelet at the
  DSR time of one scatterer at (x0, tau0) migrate to an image whose largest
  amplitude sits at (x0, tau0);
* zero offset at x = mid: t = 2 tau (the one-way tau axis, psktmCPU.c:46,78-79).

Each runs on the CPU oracle here and, marked gpu, through libktm.so.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle

V = 2000.0


def _spike_case():
    gx, gy, gz = oracle.grid(51, 20.0, 0.0), oracle.grid(1, 1.0, 0.0), oracle.grid(251, 0.001, 0.0)
    nt, dt, j0 = 200, 0.004, 100
    tr = np.zeros((1, nt), np.float32)
    tr[0, j0] = 1.0
    z = np.zeros(1, np.float32)
    mid = np.array([500.0], np.float32)
    vel = np.full(251, V, np.float32)
    return gx, gy, gz, dt, mid, z.copy(), z.copy(), z.copy(), tr, vel, j0


def _check_isochron(img, j0):
    x = 20.0 * np.arange(51)
    tau = 0.001 * np.arange(251)
    t = 2.0 * np.sqrt(tau[None, :] ** 2 + ((x[:, None] - 500.0) / V) ** 2)
    u = t / 0.004
    nzm = img[:, 0, :] != 0
    assert nzm.any()
    # every non-zero sample lies on the isochron floor(t/dt) = j0 (FP32 rounding margin)
    assert np.all((u[nzm] >= j0 - 1e-3) & (u[nzm] < j0 + 1 + 1e-3))
    # and every column within reach has at least one: the ellipse is complete
    reach = np.abs(x - 500.0) / V < 0.19
    assert np.all(nzm[reach].any(axis=1))
    # the amplitude is the reference weight |tau| sqrt(t) (samples of value 1)
    w = tau[None, :] * np.sqrt(t)
    assert np.allclose(img[:, 0, :][nzm], w[nzm], rtol=2e-5)


def _diffractor_case(nt=500, dt=0.004, x0=1000.0, tau0=0.3, f=25.0):
    mids = 12.5 * np.arange(161)
    offs = 50.0 * np.arange(11)          # half offsets 0..500 m
    mx = np.tile(mids, len(offs)).astype(np.float32)
    ox = np.repeat(offs, len(mids)).astype(np.float32)
    s = mx - ox
    r = mx + ox
    tk = np.sqrt(tau0 ** 2 + ((s - x0) / V) ** 2) + np.sqrt(tau0 ** 2 + ((r - x0) / V) ** 2)
    t = dt * np.arange(nt)
    a = (np.pi * f * (t[None, :] - tk[:, None])) ** 2
    tr = ((1.0 - 2.0 * a) * np.exp(-a)).astype(np.float32)
    gx, gy, gz = oracle.grid(81, 12.5, 500.0), oracle.grid(1, 1.0, 0.0), oracle.grid(301, 0.002, 0.0)
    z = np.zeros_like(mx)
    vel = np.full(301, V, np.float32)
    return gx, gy, gz, dt, mx, z, ox, z.copy(), tr, vel


def _check_focus(img, x0=1000.0, tau0=0.3):
    # within one grid step (the truncating pick reads the sample at or before t,
    # which moves the focus up to one tau sample later)
    i, _, l = np.unravel_index(np.argmax(np.abs(img)), img.shape)
    assert abs(500.0 + 12.5 * i - x0) <= 12.5 * 1.01
    assert abs(0.002 * l - tau0) <= 0.002 * 1.01


def test_spike_isochron_oracle():
    c = _spike_case()
    img = oracle.migrate_ref32(*c[:-1])
    _check_isochron(img, c[-1])


def test_diffractor_focus_oracle():
    c = _diffractor_case()
    _check_focus(oracle.migrate_f64(*c, pick=1, prefold=0))
    _check_focus(oracle.migrate_ref32(*c))


def test_zero_offset_two_way_time_oracle():
    # spike at j0 with dt = 2 dtau: the image peaks at tau = j0 dtau (t = 2 tau = j0 dt)
    gx, gy, gz = oracle.grid(1, 1.0, 0.0), oracle.grid(1, 1.0, 0.0), oracle.grid(64, 0.001, 0.0)
    tr = np.zeros((1, 64), np.float32)
    tr[0, 40] = 1.0
    z = np.zeros(1, np.float32)
    img = oracle.migrate_f64(gx, gy, gz, 0.002, z, z, z, z, tr, np.full(64, 1800.0, np.float32),
                             pick=1, prefold=0)
    assert np.argmax(np.abs(img[0, 0])) == 40


@pytest.mark.gpu
@pytest.mark.parametrize("entry", ["reference", "fast-truncate"])
def test_spike_isochron_gpu(cuda, ktm_lib, entry):
    import ktm
    gx, gy, gz, dt, mx, my, ox, oy, tr, vel, j0 = _spike_case()
    if entry == "reference":
        img = ktm.ktmMigrationGPU(gx, gy, gz, (1, tr.shape[1], dt), mx, my, ox, oy, tr, vel)
    else:
        img = ktm.migrate(imageX=gx, imageY=gy, imageZ=gz, dt=dt, midX=mx, midY=my, offX=ox,
                          offY=oy, traces=tr, velocity=vel, pick="truncate", weight="sqrt")
    _check_isochron(np.asarray(img).reshape(51, 1, 251), j0)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(mode="reference", pick="truncate"),
                                dict(pick="linear"),
                                dict(pick="linear", weight="prefold", pack_format="f16")])
def test_diffractor_focus_gpu(cuda, ktm_lib, kw):
    import ktm
    gx, gy, gz, dt, mx, my, ox, oy, tr, vel = _diffractor_case()
    img = ktm.migrate(imageX=gx, imageY=gy, imageZ=gz, dt=dt, midX=mx, midY=my, offX=ox, offY=oy,
                      traces=tr, velocity=vel, **kw)
    _check_focus(np.asarray(img))
