"""IBM-32 ingest on the device and the psktm driver end to end (needs a B200).

* ktmIBM32toIEEE / ktmIBM32toIEEEDevice bit-identical to the reference's
  ktmIBM32toIEEE (golden words incl. zero, infinities, the 0 * inf NaN,
  subnormals) and to the oracle on ten million random words, aligned and
  misaligned buffers;
* IBM words as raw traces of a job: reference mode bit-identical to the
  oracle on the decoded floats; fast mode (conversion fused into the rho /
  pack pass) identical to the same job given the decoded floats;
* psktm on a data directory written in the Octave writers' layout:
  reference mode bit-identical to the oracle, fast mode with rebased UTM-size
  coordinates within the accuracy gate of the FP64 oracle.
"""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import load_golden
from ktm import io as kio
from ktm.synth import encode_ibm32

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PSKTM = os.path.join(ROOT, "seismic-migration_b200", "ktm", "psktm")


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_ibm_host_entry_bit_identical_to_reference_golden(cuda, ktm_lib):
    g = load_golden("ref_ibm32.npz")
    out = kio.ibm32_to_ieee(g["words"])
    assert np.array_equal(_bits(out), _bits(g["ieee"]))


@pytest.mark.parametrize("offset", [0, 1, 3])
def test_ibm_device_entry_bit_identical(cuda, ktm_lib, offset):
    import torch
    g = load_golden("ref_ibm32.npz")
    w = torch.as_tensor(g["words"].view(np.int32)).to(cuda)
    out = kio.ibm32_to_ieee(w[offset:])          # offset 1, 3: the unaligned scalar path
    torch.cuda.synchronize()
    assert np.array_equal(_bits(out.cpu().numpy()), _bits(g["ieee"][offset:]))


def test_ibm_device_large_random_matches_oracle(cuda, ktm_lib):
    import torch
    rng = np.random.default_rng(11)
    words = rng.integers(0, 2**32, 10_000_003, dtype=np.uint64).astype(np.uint32)
    out = kio.ibm32_to_ieee(torch.as_tensor(words.view(np.int32)).to(cuda)).cpu().numpy()
    ref = oracle.ibm32_to_ieee(words)
    assert np.array_equal(_bits(out), _bits(ref))


def _case(seed, ntr=61, nt=150, nx=5, ny=4, nz=90, dt=0.004):
    rng = np.random.default_rng(seed)
    gx, gy, gz = oracle.grid(nx, 30.0, -60.0), oracle.grid(ny, 25.0, -40.0), oracle.grid(nz, 0.00173, 0.0)
    mid = rng.uniform(-300, 300, (ntr, 2)).astype(np.float32)
    off = rng.uniform(-300, 300, (ntr, 2)).astype(np.float32)
    tr = (rng.standard_normal((ntr, nt)) * 50.0).astype(np.float32)
    words = encode_ibm32(tr)
    vel = np.linspace(1500.0, 3000.0, nz).astype(np.float32)
    return gx, gy, gz, dt, mid, off, words, vel


def test_reference_mode_ibm_traces_bit_identical(cuda, ktm_lib):
    import ktm
    gx, gy, gz, dt, mid, off, words, vel = _case(21)
    img = ktm.migrate(imageX=gx, imageY=gy, imageZ=gz, dt=dt, midX=mid[:, 0], midY=mid[:, 1],
                      offX=off[:, 0], offY=off[:, 1], traces=words, velocity=vel,
                      mode="reference", pick="truncate")
    ref = oracle.migrate_ref32(gx, gy, gz, dt, mid[:, 0], mid[:, 1], off[:, 0], off[:, 1],
                               oracle.ibm32_to_ieee(words), vel)
    assert np.array_equal(_bits(img), _bits(ref))


@pytest.mark.parametrize("rho,fmt", [(0, "f32"), (3, "f16"), (2, "bf16")])
def test_fast_mode_ibm_fused_prep_equals_decoded_input(cuda, ktm_lib, rho, fmt):
    import ktm
    import torch
    gx, gy, gz, dt, mid, off, words, vel = _case(22)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to(cuda)  # noqa: E731
    common = dict(imageX=gx, imageY=gy, imageZ=gz, dt=dt, midX=t(mid[:, 0]), midY=t(mid[:, 1]),
                  offX=t(off[:, 0]), offY=t(off[:, 1]), velocity=t(vel), mode="fast",
                  pick="linear", rho=rho, pack_format=fmt)
    a = ktm.migrate(traces=t(words.view(np.int32)), **common)
    b = ktm.migrate(traces=t(oracle.ibm32_to_ieee(words)), **common)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_prepare_takes_ibm_words(cuda, ktm_lib):
    import ktm
    import torch
    words = encode_ibm32(np.random.default_rng(23).standard_normal((9, 77)).astype(np.float32))
    a = ktm.prepare(torch.as_tensor(words.view(np.int32)).to(cuda), 0.004, fmt="f16", rho=3,
                    prefold=False)
    b = ktm.prepare(torch.as_tensor(oracle.ibm32_to_ieee(words)).to(cuda), 0.004, fmt="f16",
                    rho=3, prefold=False)
    assert torch.equal(a.data, b.data) and torch.equal(a.scale, b.scale)


def _write_dir(path, seed, base=0.0, ntr=80, nt=200, nx=6, ny=3, nz=120):
    rng = np.random.default_rng(seed)
    sx = (base + rng.uniform(0, 600, ntr)).astype(np.float32)
    sy = (base + rng.uniform(0, 300, ntr)).astype(np.float32)
    rx = (base + rng.uniform(0, 600, ntr)).astype(np.float32)
    ry = (base + rng.uniform(0, 300, ntr)).astype(np.float32)
    from test_parity_gpu import band_limited
    tr = band_limited(rng, ntr, nt, 0.004) * 100.0
    inp = kio.Inp(nt, 0.004, ntr, (nx, 40.0, base + 200.0), (ny, 50.0, base + 100.0),
                  (nz, 0.00173, 0.0))
    vel = np.linspace(1600.0, 2800.0, nz).astype(np.float32)
    kio.write_survey(str(path), inp, encode_ibm32(tr), sx, sy, rx, ry, vel)
    return inp, sx, sy, rx, ry, tr, vel


@pytest.mark.skipif(not os.path.exists(PSKTM), reason="psktm not built")
def test_psktm_reference_mode_bit_identical(cuda, ktm_lib, tmp_path):
    inp, sx, sy, rx, ry, tr, vel = _write_dir(tmp_path, 31)
    r = subprocess.run([PSKTM, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    img = kio.read_image(str(tmp_path / "outputData.bin"), inp)
    sv = kio.load_survey(str(tmp_path))
    gx, gy, gz = sv.grids()
    ref = oracle.migrate_ref32(gx, gy, gz, inp.sampleRate, sv.midX, sv.midY, sv.offX, sv.offY,
                               oracle.ibm32_to_ieee(sv.traces), sv.velocity)
    assert np.array_equal(_bits(img), _bits(ref))


@pytest.mark.skipif(not os.path.exists(PSKTM), reason="psktm not built")
def test_psktm_fast_mode_rebased_utm_coordinates(cuda, ktm_lib, tmp_path):
    """Coordinates near 500 km: float32 spacing there is 1/32 m.  Rebased in
    FP64 (the default in fast mode) the migration meets the 1e-3 gate against
    the FP64 oracle (reference weight) on the rebased geometry."""
    inp, sx, sy, rx, ry, tr, vel = _write_dir(tmp_path, 32, base=500000.0)
    out = tmp_path / "fast.bin"
    r = subprocess.run([PSKTM, "--mode", "fast", "--format", "f32", "-o", str(out), str(tmp_path)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    img = kio.read_image(str(out), inp)
    sv = kio.load_survey(str(tmp_path), rebase=True)
    gx, gy, gz = sv.grids()
    ref = oracle.migrate_f64(gx, gy, gz, inp.sampleRate, sv.midX, sv.midY, sv.offX, sv.offY,
                             oracle.ibm32_to_ieee(sv.traces), sv.velocity, pick=1, prefold=False)
    err = float(np.linalg.norm(img - ref) / np.linalg.norm(ref))
    assert err < 1e-3, err


def test_ibm_device_all_words_exhaustive(cuda, ktm_lib):
    """Every one of the 2^32 IBM-32 words: the device conversion is bit-identical
    to the reference's own ktmIBM32toIEEE (compiled from its sources into
    oracle/_ref) or, where that was not built, to the oracle restatement."""
    import concurrent.futures as cf
    import os as _os

    import torch
    from ktm import io as kio
    conv = oracle.ibm32_to_ieee_reference_c if oracle.ref_available() else oracle.ibm32_to_ieee
    n = 1 << 28
    parts = max(1, min(32, _os.cpu_count() or 1))
    with cf.ThreadPoolExecutor(parts) as ex:       # the C conversion releases the GIL
        for k in range(16):
            w64 = torch.arange(k * n, (k + 1) * n, device=cuda, dtype=torch.int64)
            w = torch.where(w64 >= 2**31, w64 - 2**32, w64).to(torch.int32)
            del w64
            got = kio.ibm32_to_ieee(w).view(torch.int32).cpu().numpy()
            words = w.cpu().numpy().view(np.uint32)
            del w
            ref = np.concatenate(list(ex.map(conv, np.array_split(words, parts)))).view(np.int32)
            bad = np.flatnonzero(got != ref)
            assert bad.size == 0, (k, hex(int(words[bad[0]])), hex(got[bad[0]]), hex(ref[bad[0]]))
