"""The reference's on-disk formats through libktm.so's host readers (no GPU).

inp.txt as ktmWriteTraceBlockConstOffset.m:154-167 writes it ("%f " per
value), inputData.bin as IBM words or float32, the source/receiver files and
the midpoint/half-offset conversion of ktmConvertXYtoOffMid.m:12 (FP64, then
float), velModel.bin 1-D and cube, outputData.bin, error paths, and the psktm
driver's argument handling.
"""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import oracle
from ktm import io as kio
from ktm._lib import KTM_ERR_IO, KtmError
from ktm.synth import encode_ibm32

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PSKTM = os.path.join(ROOT, "seismic-migration_b200", "ktm", "psktm")


def _inp(ntr=7, nt=33, nx=4, ny=3, nz=17):
    return kio.Inp(nt, 0.004, ntr, (nx, 25.0, 100.0), (ny, 12.5, -50.0), (nz, 0.004, 0.0))


def _survey(rng, ntr=7, nt=33, base=0.0):
    sx = (base + rng.uniform(0, 1000, ntr)).astype(np.float32)
    sy = (base + rng.uniform(0, 1000, ntr)).astype(np.float32)
    rx = (base + rng.uniform(0, 1000, ntr)).astype(np.float32)
    ry = (base + rng.uniform(0, 1000, ntr)).astype(np.float32)
    tr = rng.standard_normal((ntr, nt)).astype(np.float32)
    return sx, sy, rx, ry, tr


def test_inp_round_trip_and_octave_layout(ktm_lib, tmp_path):
    inp = _inp()
    p = str(tmp_path / "inp.txt")
    kio.write_inp(p, inp)
    text = open(p).read()
    assert len(text.split()) == 12 and text.startswith("33.000000 0.004000 7.000000 ")
    back = kio.read_inp(p)
    assert back == kio.Inp(33, np.float32(0.004).item(), 7, (4, 25.0, 100.0), (3, 12.5, -50.0),
                           (17, np.float32(0.004).item(), 0.0))


def test_inp_written_by_octave_is_read(ktm_lib, tmp_path):
    # the Octave writer's format: "%f " after every value, newline-free
    p = tmp_path / "inp.txt"
    p.write_text("1001.000000 0.004000 2048.000000 0.000000 12.500000 256.000000 "
                 "0.000000 1.000000 1.000000 0.000000 0.004000 1001.000000 ")
    inp = kio.read_inp(str(p))
    assert (inp.tracePts, inp.traceNo) == (1001, 2048)
    assert inp.x == (256, 12.5, 0.0) and inp.y == (1, 1.0, 0.0)
    assert inp.z[0] == 1001 and abs(inp.z[1] - 0.004) < 1e-9


def test_inp_too_few_numbers_is_an_io_error(ktm_lib, tmp_path):
    p = tmp_path / "inp.txt"
    p.write_text("1 2 3 4 5 6 7 8 9 10 11")
    with pytest.raises(KtmError) as e:
        kio.read_inp(str(p))
    assert e.value.code == KTM_ERR_IO


@pytest.mark.parametrize("ibm", [False, True])
def test_survey_round_trip_float_and_ibm(ktm_lib, tmp_path, ibm):
    rng = np.random.default_rng(3)
    sx, sy, rx, ry, tr = _survey(rng)
    inp = _inp()
    words = encode_ibm32(tr) if ibm else tr
    vel = np.linspace(1500, 2500, 17).astype(np.float32)
    kio.write_survey(str(tmp_path), inp, words, sx, sy, rx, ry, vel)
    sv = kio.load_survey(str(tmp_path), ibm=ibm)
    assert sv.fmt == ("ibm32" if ibm else "f32")
    assert np.array_equal(sv.traces.view(np.uint32), np.asarray(words).view(np.uint32))
    # ktmConvertXYtoOffMid.m:12 in FP64, rounded once to float
    f64 = lambda a: a.astype(np.float64)  # noqa: E731
    assert np.array_equal(sv.midX, ((f64(rx) + f64(sx)) / 2).astype(np.float32))
    assert np.array_equal(sv.midY, ((f64(ry) + f64(sy)) / 2).astype(np.float32))
    assert np.array_equal(sv.offX, ((f64(rx) - f64(sx)) / 2).astype(np.float32))
    assert np.array_equal(sv.offY, ((f64(ry) - f64(sy)) / 2).astype(np.float32))
    assert np.array_equal(sv.velocity, vel) and sv.origin == (0.0, 0.0)


def test_survey_rebase_shifts_coordinates_and_axes(ktm_lib, tmp_path):
    rng = np.random.default_rng(4)
    sx, sy, rx, ry, tr = _survey(rng, base=500000.0)
    inp = kio.Inp(33, 0.004, 7, (4, 25.0, 500100.0), (3, 12.5, 500050.0), (17, 0.004, 0.0))
    kio.write_survey(str(tmp_path), inp, tr, sx, sy, rx, ry, np.full(17, 2000.0, np.float32))
    sv = kio.load_survey(str(tmp_path), ibm=False, rebase=True)
    ox = np.floor(min(sx.min(), rx.min()))
    oy = np.floor(min(sy.min(), ry.min()))
    assert sv.origin == (float(ox), float(oy))
    f64 = lambda a: a.astype(np.float64)  # noqa: E731
    assert np.array_equal(sv.midX, ((f64(rx) + f64(sx)) / 2 - ox).astype(np.float32))
    assert sv.inp.x[2] == np.float32(np.float32(500100.0) - ox)
    assert sv.inp.y[2] == np.float32(np.float32(500050.0) - oy)


def test_velocity_cube_detected(ktm_lib, tmp_path):
    rng = np.random.default_rng(5)
    sx, sy, rx, ry, tr = _survey(rng)
    vel = rng.uniform(1500, 3000, (4, 3, 17)).astype(np.float32)
    kio.write_survey(str(tmp_path), _inp(), tr, sx, sy, rx, ry, vel)
    sv = kio.load_survey(str(tmp_path), ibm=False)
    assert sv.velocity.shape == (4, 3, 17) and np.array_equal(sv.velocity, vel)


@pytest.mark.parametrize("damage", ["missing", "short_data", "short_vel"])
def test_survey_errors_are_io_errors(ktm_lib, tmp_path, damage):
    rng = np.random.default_rng(6)
    sx, sy, rx, ry, tr = _survey(rng)
    kio.write_survey(str(tmp_path), _inp(), tr, sx, sy, rx, ry, np.full(17, 2000.0, np.float32))
    if damage == "missing":
        os.remove(tmp_path / "inputRecY.bin")
    elif damage == "short_data":
        tr[:-1].tofile(tmp_path / "inputData.bin")
    else:
        np.full(5, 2000.0, np.float32).tofile(tmp_path / "velModel.bin")
    with pytest.raises(KtmError) as e:
        kio.load_survey(str(tmp_path), ibm=False)
    assert e.value.code == KTM_ERR_IO


def test_image_write_read(ktm_lib, tmp_path):
    img = np.random.default_rng(7).standard_normal((4, 3, 17)).astype(np.float32)
    p = str(tmp_path / "outputData.bin")
    kio.write_image(p, img)
    assert np.array_equal(kio.read_image(p, _inp()), img)


def test_ibm_encoder_decodes_through_the_reference_arithmetic():
    """encode_ibm32 (synthetic IBM data) inverts the reference's decoder up to
    its rounding and the FRACTION_MASK bias (2^-24 relative)."""
    x = np.random.default_rng(8).standard_normal(5000).astype(np.float32) * 1e3
    x[:3] = [0.0, 1.0, -100.0]
    back = oracle.ibm32_to_ieee(encode_ibm32(x))
    assert back[0] == 0.0
    assert np.max(np.abs(back - x) / np.maximum(np.abs(x), 1e-30))[()] < 2.5e-6


@pytest.mark.skipif(not os.path.exists(PSKTM), reason="psktm not built")
def test_psktm_usage_and_missing_directory(ktm_lib, tmp_path):
    r = subprocess.run([PSKTM], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr
    r = subprocess.run([PSKTM, "--mode", "nonsense", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 1
    r = subprocess.run([PSKTM, str(tmp_path / "absent")], capture_output=True, text=True)
    assert r.returncode == 2 and "inp.txt" in r.stderr
