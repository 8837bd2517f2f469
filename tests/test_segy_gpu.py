"""Time-axis interpolation on the device and SEG-Y input to psktm (needs a B200).

* ktmInterpTraces is bit-identical to the restatement of ktmInterpTraceBlock.m
  opt 2 (FP64 interp1, rounded to float): levels 0..5, one- and two-sample
  traces, a strided output, more traces than one launch row holds (65,535);
* migrating traces upsampled by 2^N with the reference's truncating pick
  approaches the linear pick on the original traces as N grows (the use the
  reference's pre-processing had for the interpolation);
* psktm --segy: the same image, bit for bit, as psktm on the same traces and
  coordinates written in the directory format; a negative (divisor) coordinate
  scalar is honoured.
"""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import oracle
import segy as oseg
from ktm import io as kio
from ktm.synth import encode_ibm32
from test_parity_gpu import band_limited, rel_l2

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PSKTM = os.path.join(ROOT, "seismic-migration_b200", "ktm", "psktm")


@pytest.mark.parametrize("levels", [0, 1, 2, 3, 5])
def test_interp_bit_identical(cuda, ktm_lib, levels):
    import ktm
    import torch
    x = np.random.default_rng(levels).standard_normal((37, 129)).astype(np.float32) * 1e3
    y = ktm.interp_time(torch.as_tensor(x).to(cuda), levels).cpu().numpy()
    assert np.array_equal(y.view(np.uint32), oseg.interp1_linear(x, levels).view(np.uint32))


def test_interp_edges_strided_and_many_traces(cuda, ktm_lib):
    import ktm
    import torch
    rng = np.random.default_rng(9)
    for nt in (1, 2):
        x = rng.standard_normal((5, nt)).astype(np.float32)
        y = ktm.interp_time(torch.as_tensor(x).to(cuda), 3).cpu().numpy()
        assert np.array_equal(y, oseg.interp1_linear(x, 3))
    x = rng.standard_normal((70000, 24)).astype(np.float32)
    nout = 23 * 4 + 1
    buf = torch.full((70000, nout + 5), 7.0, device=cuda)
    out = ktm.interp_time(torch.as_tensor(x).to(cuda), 2, out=buf[:, :nout])
    assert out.stride(0) == nout + 5
    assert np.array_equal(buf[:, :nout].cpu().numpy(), oseg.interp1_linear(x, 2))
    assert bool((buf[:, nout:] == 7.0).all())


def test_upsampled_truncation_approaches_linear_pick(cuda, ktm_lib):
    import ktm
    import torch
    rng = np.random.default_rng(10)
    ntr, nt, dt = 120, 200, 0.004
    gx, gy, gz = oracle.grid(6, 30.0, -90.0), oracle.grid(2, 40.0, 0.0), oracle.grid(180, 0.002, 0.0)
    mx = rng.uniform(-200, 200, ntr).astype(np.float32)
    my = rng.uniform(-50, 50, ntr).astype(np.float32)
    ox = rng.uniform(-300, 300, ntr).astype(np.float32)
    oy = rng.uniform(-100, 100, ntr).astype(np.float32)
    tr = band_limited(rng, ntr, nt, dt)
    vel = np.linspace(1600, 2600, 180).astype(np.float32)
    ref = oracle.migrate_f64(gx, gy, gz, dt, mx, my, ox, oy, tr, vel, pick=1, prefold=0)
    errs = []
    for n in (1, 2, 4):
        up = ktm.interp_time(torch.as_tensor(tr).to(cuda), n).cpu().numpy()
        img = ktm.ktmMigrationGPU(gx, gy, gz, (ntr, up.shape[1], dt / 2 ** n), mx, my, ox, oy,
                                  up, vel)
        errs.append(rel_l2(np.asarray(img), ref))
    assert errs[2] < errs[1] < errs[0]
    assert errs[2] < 0.05


def _survey_files(tmp_path, scalar):
    rng = np.random.default_rng(11)
    ntr, ns = 90, 220
    s = np.stack([rng.integers(0, 800, ntr), rng.integers(0, 400, ntr)], 1)
    r = np.stack([rng.integers(0, 800, ntr), rng.integers(0, 400, ntr)], 1)
    tr = band_limited(rng, ntr, ns, 0.004) * 50.0
    words = encode_ibm32(tr)
    h = np.zeros((ntr, 101), np.int64)
    h[:, 20] = scalar
    mul = float(-scalar) if scalar < 0 else 1.0
    h[:, 21:23] = (s * mul).astype(np.int64)
    h[:, 23:25] = (r * mul).astype(np.int64)
    seg = tmp_path / "line.segy"
    oseg.write_segy(str(seg), words, 1, 4000, h, "C 1 TEST LINE")
    inp = kio.Inp(ns, 0.004, ntr, (8, 50.0, 200.0), (3, 100.0, 100.0), (150, 0.002, 0.0))
    vel = np.linspace(1700.0, 2500.0, 150).astype(np.float32)
    kio.write_survey(str(tmp_path), inp, words, s[:, 0], s[:, 1], r[:, 0], r[:, 1], vel)
    return seg, inp


@pytest.mark.skipif(not os.path.exists(PSKTM), reason="psktm not built")
@pytest.mark.parametrize("scalar", [1, -100])
def test_psktm_segy_matches_directory_input(cuda, ktm_lib, tmp_path, scalar):
    seg, inp = _survey_files(tmp_path, scalar)
    a = tmp_path / "a.bin"
    b = tmp_path / "b.bin"
    r1 = subprocess.run([PSKTM, "-o", str(a), str(tmp_path)], capture_output=True, text=True,
                        timeout=300)
    r2 = subprocess.run([PSKTM, "--segy", str(seg), "-o", str(b), str(tmp_path)],
                        capture_output=True, text=True, timeout=300)
    assert r1.returncode == 0 and r2.returncode == 0, r1.stderr + r2.stderr
    ia, ib = kio.read_image(str(a), inp), kio.read_image(str(b), inp)
    assert np.abs(ia).max() > 0
    # integer coordinates (times the scalar): the same floats either way
    assert np.array_equal(ia.view(np.uint32), ib.view(np.uint32))
