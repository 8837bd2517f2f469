"""SEG-Y reader (ktm_segy.c) against the restatement of the Octave front end
(oracle/segy.py), and the time-interpolation oracle's known answers (no GPU).

No SEG-Y data ships with the reference or this container, so the files are
written here: every sample format the reader takes (1 IBM, 2 int32, 3 int16,
5 IEEE, 8 int8), big- and little-endian, positive / negative / zero coordinate
scalars, ragged trace ranges, damaged files.
"""
from __future__ import annotations

import numpy as np
import pytest

import segy as oseg
from ktm import io as kio
from ktm._lib import KTM_ERR_ARG, KTM_ERR_IO, KtmError
from ktm.synth import encode_ibm32

TEXT = "C 1 CLIENT ACME  LINE 42  AREA X/Y: 500000#4100000 @ UTM {ZONE} ~ END"


def _headers(rng, ntr, scalar=-100, negative=False):
    h = rng.integers(0, 30000, (ntr, 101)).astype(np.int64)
    h[:, 20] = scalar
    lo = -400000 if negative else 0
    h[:, 21:25] = rng.integers(lo, 50_000_000, (ntr, 4))
    return h


def _samples(rng, fmt, ntr, ns):
    x = rng.standard_normal((ntr, ns)).astype(np.float32)
    if fmt == 1:
        return encode_ibm32(x)
    if fmt == 2:
        return (x * 1e6).astype(np.int32)
    if fmt == 3:
        return (x * 3000).astype(np.int16)
    if fmt == 8:
        return (x * 40).clip(-128, 127).astype(np.int8)
    return x


@pytest.mark.parametrize("fmt", [1, 2, 3, 5, 8])
@pytest.mark.parametrize("big", [True, False])
def test_reader_matches_script_decoding(ktm_lib, tmp_path, fmt, big):
    rng = np.random.default_rng(fmt * 7 + big)
    ntr, ns = 23, 37
    smp = _samples(rng, fmt, ntr, ns)
    hdr = _headers(rng, ntr, scalar=10)
    path = str(tmp_path / "a.segy")
    oseg.write_segy(path, smp, fmt, 4000, hdr, TEXT, big_endian=big)
    raw = open(path, "rb").read()
    info, s, th = kio.read_segy(path, first=3, count=15, big_endian=big)
    assert (info.samplesPerTrace, info.sampleInterval, info.format, info.traceCount) == (ns, 4000, fmt, ntr)
    assert info.text.decode().split("\n") == oseg.script_text(raw).split("\n")
    if big:   # the script assembles the reel header big-endian whatever the file's order
        assert list(info.reel32) + list(info.reel16) == oseg.script_reel_header(raw)
    if fmt != 8:
        ref = oseg.script_samples(raw, ns, fmt, big, 3, 15)
        if fmt in (1, 5):
            assert np.array_equal(s.view(np.uint32), ref.astype(np.uint32))
        else:
            assert np.array_equal(s, ref.astype(np.float32))
    else:
        assert np.array_equal(s, smp[3:18].astype(np.float32))
    sh = oseg.script_trace_headers(raw, ns, {1: 4, 2: 4, 3: 2, 5: 4, 8: 1}[fmt], big, 3, 15)
    got = np.array([list(t.values) for t in th])
    assert np.array_equal(got, sh)             # non-negative fields: same as the script
    assert np.array_equal(got, hdr[3:18])
    x = np.array([[t.srcX, t.srcY, t.recX, t.recY] for t in th])
    assert np.array_equal(x, hdr[3:18, 21:25] * 10.0)


def test_negative_fields_and_divisor_scalar(ktm_lib, tmp_path):
    """Negative coordinates and the divisor scalar -100: decoded as two's
    complement (the script's int32()/int16() casts saturate them instead)."""
    rng = np.random.default_rng(3)
    hdr = _headers(rng, 9, scalar=-100, negative=True)
    hdr[:, 0] = -5
    path = str(tmp_path / "n.segy")
    oseg.write_segy(path, _samples(rng, 5, 9, 11), 5, 2000, hdr)
    _, _, th = kio.read_segy(path)
    got = np.array([list(t.values) for t in th])
    assert np.array_equal(got, hdr)
    x = np.array([[t.srcX, t.srcY, t.recX, t.recY] for t in th])
    assert np.array_equal(x, hdr[:, 21:25] / 100.0)
    sat = oseg.script_trace_headers(open(path, "rb").read(), 11, 4, True, 0, 9)
    assert (sat[:, 20] == 32767).all() and (sat[:, 0] == 2**31 - 1).all()


def test_zero_scalar_means_one(ktm_lib, tmp_path):
    rng = np.random.default_rng(4)
    hdr = _headers(rng, 4, scalar=0)
    path = str(tmp_path / "z.segy")
    oseg.write_segy(path, _samples(rng, 3, 4, 8), 3, 1000, hdr)
    _, _, th = kio.read_segy(path)
    assert np.array_equal(np.array([[t.srcX, t.srcY, t.recX, t.recY] for t in th]), hdr[:, 21:25])


@pytest.mark.parametrize("rebase", [False, True])
def test_segy_survey_mid_offset(ktm_lib, tmp_path, rebase):
    rng = np.random.default_rng(5)
    ntr, ns = 31, 50
    hdr = _headers(rng, ntr, scalar=-100)
    words = _samples(rng, 1, ntr, ns)
    path = str(tmp_path / "s.segy")
    oseg.write_segy(path, words, 1, 2000, hdr)
    sv = kio.load_segy_survey(path, first=2, count=25, rebase=rebase)
    assert sv.fmt == "ibm32" and np.array_equal(sv.traces, words[2:27])
    assert sv.inp.tracePts == ns and sv.inp.traceNo == 25
    assert abs(sv.inp.sampleRate - 0.002) < 1e-9
    c = hdr[2:27, 21:25] / 100.0
    sx, sy, rx, ry = c.T
    ox = np.floor(min(sx.min(), rx.min())) if rebase else 0.0
    oy = np.floor(min(sy.min(), ry.min())) if rebase else 0.0
    assert sv.origin == (ox, oy)
    assert np.array_equal(sv.midX, ((rx + sx) / 2 - ox).astype(np.float32))
    assert np.array_equal(sv.midY, ((ry + sy) / 2 - oy).astype(np.float32))
    assert np.array_equal(sv.offX, ((rx - sx) / 2).astype(np.float32))
    assert np.array_equal(sv.offY, ((ry - sy) / 2).astype(np.float32))


def test_segy_errors(ktm_lib, tmp_path):
    rng = np.random.default_rng(6)
    path = str(tmp_path / "e.segy")
    oseg.write_segy(path, _samples(rng, 5, 5, 10), 5, 1000)
    raw = open(path, "rb").read()
    with pytest.raises(KtmError) as e:
        kio.read_segy(path, first=3, count=5)
    assert e.value.code == KTM_ERR_ARG
    open(tmp_path / "short.segy", "wb").write(raw[:3000])
    with pytest.raises(KtmError) as e:
        kio.segy_open(str(tmp_path / "short.segy"))
    assert e.value.code == KTM_ERR_IO
    bad = bytearray(raw)
    bad[3225] = 7                                 # sample format 7: not read
    open(tmp_path / "fmt.segy", "wb").write(bytes(bad))
    with pytest.raises(KtmError) as e:
        kio.segy_open(str(tmp_path / "fmt.segy"))
    assert e.value.code == KTM_ERR_IO
    # a partial last trace is not counted
    open(tmp_path / "cut.segy", "wb").write(raw[:-7])
    assert kio.segy_open(str(tmp_path / "cut.segy")).traceCount == 4


# ------------------------------------------------------------ interpolation oracle ----
def test_interp_oracle_known_answers():
    t = np.arange(12, dtype=np.float64)
    lin = (3.0 * t - 7.0)[None, :].astype(np.float32)
    for n in range(5):
        y = oseg.interp1_linear(lin, n)
        assert y.shape == (1, 11 * 2 ** n + 1)
        tt = np.arange(y.shape[1]) / 2.0 ** n
        assert np.array_equal(y[0], (3.0 * tt - 7.0).astype(np.float32))
    x = np.random.default_rng(7).standard_normal((3, 9)).astype(np.float32)
    y = oseg.interp1_linear(x, 3)
    assert np.array_equal(y[:, ::8], x)                     # knots kept
    assert np.array_equal(oseg.interp1_linear(x, 0), x)
    assert np.array_equal(oseg.interp1_linear(x[:, :1], 2), x[:, :1])
