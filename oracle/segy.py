"""Oracle for the SEG-Y reader and the time-axis interpolation (test
infrastructure: only tests and the bench's CPU legs use it).

Restates, in numpy, what the Octave front end computes:
- ``script_reel_header``: ktmGetInputMeta.m opt 2 (:54-68): three 32-bit and 24
  16-bit reel fields, assembled from the bytes in file order (big-endian,
  unsigned, whatever endianness is asked for);
- ``script_trace_headers``: ktmGetInputMeta.m opt 3 (:126-132): the 240-byte
  header as 16-bit words of the file's endianness, pairs joined into 32-bit
  values, then Octave's int32() / int16() casts, which SATURATE (a negative
  value stored in two's complement becomes 2^31-1 / 2^15-1);
- ``script_text``: the EBCDIC table of ktmGetInputMeta.m:30-45;
- ``script_samples``: ktmGetInputTrace.m:33-72 (uint32 words for formats 1 and
  the rest, int32 for 2, int16 for 3);
- ``interp1_linear``: ktmInterpTraceBlock.m:134-154 with Octave's interp1
  'linear', y = (y[i+1] - y[i]) * (t - i) + y[i] in double.

Octave is not installed, so these are pinned by known answers in the tests
(parity unpinned beyond them), and ``write_segy`` makes the test files.
"""
from __future__ import annotations

import numpy as np

# EBCDIC -> ASCII as the script's table (1-based tbl(b) for byte value b)
_TBL = np.full(256, ord("?"), np.uint8)
for _i, _c in enumerate("abcdefghi"):
    _TBL[129 + _i] = ord(_c)
for _i, _c in enumerate("jklmnopqr"):
    _TBL[145 + _i] = ord(_c)
for _i, _c in enumerate("~stuvwxyz"):
    _TBL[161 + _i] = ord(_c)
for _i, _c in enumerate("{ABCDEFGHI"):
    _TBL[192 + _i] = ord(_c)
for _i, _c in enumerate("}JKLMNOPQR"):
    _TBL[208 + _i] = ord(_c)
for _i, _c in enumerate("\\ STUVWXYZ"):          # tbl(225) is NUL in the script; space here
    _TBL[224 + _i] = ord(_c)
for _i, _c in enumerate("0123456789"):
    _TBL[240 + _i] = ord(_c)
_TBL[96], _TBL[97], _TBL[64] = ord("-"), ord("/"), ord(" ")
_TBL[122], _TBL[123], _TBL[124] = ord(":"), ord("#"), ord("@")

_ASCII_TO_EBCDIC = {int(v): k for k, v in enumerate(_TBL) if v != ord("?")}
_ASCII_TO_EBCDIC[ord(" ")] = 64


def script_text(raw: bytes) -> str:
    rows = _TBL[np.frombuffer(raw[:3200], np.uint8)].reshape(40, 80)
    return "\n".join(bytes(r).decode("ascii") for r in rows)


def script_reel_header(raw: bytes) -> list[int]:
    b = np.frombuffer(raw[3200:3600], np.uint8).astype(np.int64)
    out = [int((b[4 * i] << 24) | (b[4 * i + 1] << 16) | (b[4 * i + 2] << 8) | b[4 * i + 3])
           for i in range(3)]
    out += [int((b[12 + 2 * i] << 8) | b[13 + 2 * i]) for i in range(24)]
    return out


def _sat(v, bits):
    hi = (1 << (bits - 1)) - 1
    return np.minimum(v, hi)


def script_trace_headers(raw: bytes, ns: int, sbytes: int, big_endian: bool, first: int,
                         count: int) -> np.ndarray:
    """[count, 101] as the script returns them (saturating casts included)."""
    tb = 240 + ns * sbytes
    dt = ">u2" if big_endian else "<u2"
    rows = []
    for k in range(first, first + count):
        w = np.frombuffer(raw[3600 + k * tb: 3600 + k * tb + 240], dt).astype(np.int64)
        def join(a, b):
            return (a << 16) + b if big_endian else a + (b << 16)
        v = []
        v += [_sat(join(w[2 * i], w[2 * i + 1]), 32) for i in range(7)]
        v += [_sat(w[14 + i], 16) for i in range(4)]
        v += [_sat(join(w[18 + 2 * i], w[19 + 2 * i]), 32) for i in range(8)]
        v += [_sat(w[34 + i], 16) for i in range(2)]
        v += [_sat(join(w[36 + 2 * i], w[37 + 2 * i]), 32) for i in range(4)]
        v += [_sat(w[44 + i], 16) for i in range(76)]
        rows.append(v)
    return np.array(rows, np.int64).reshape(count, 101)


def script_samples(raw: bytes, ns: int, fmt: int, big_endian: bool, first: int, count: int):
    e = ">" if big_endian else "<"
    dt = {2: e + "i4", 3: e + "i2"}.get(fmt, e + "u4")
    sb = np.dtype(dt).itemsize
    tb = 240 + ns * sb
    out = np.empty((count, ns), np.dtype(dt).newbyteorder("="))
    for k in range(count):
        o = 3600 + (first + k) * tb + 240
        out[k] = np.frombuffer(raw[o: o + ns * sb], dt)
    return out


def write_segy(path, samples, fmt: int, dt_us: int, headers=None, text: str = "",
               big_endian: bool = True):
    """A SEG-Y rev 0 file: EBCDIC text, binary reel header (interval, samples,
    format), per trace a 240-byte header from ``headers`` ([ntr, 101] in the
    script's grouping, signed values, two's complement) and the samples (uint32
    IBM words for format 1, float32 for 5, int32 for 2, int16 for 3, int8 for 8)."""
    e = ">" if big_endian else "<"
    samples = np.asarray(samples)
    ntr, ns = samples.shape
    txt = (text + " " * 3200)[:3200]
    tb = bytes(_ASCII_TO_EBCDIC.get(ord(c), 0x6F) for c in txt)
    reel = np.zeros(3, e + "u4").tobytes()
    r16 = np.zeros(24, e + "u2")
    r16[2], r16[3], r16[4], r16[5], r16[6] = dt_us, dt_us, ns, ns, fmt
    reel += r16.tobytes() + bytes(400 - 12 - 48)
    sdt = {1: "u4", 2: "i4", 3: "i2", 5: "f4", 8: "i1"}[fmt]
    body = []
    for k in range(ntr):
        h = np.zeros(101, np.int64) if headers is None else np.asarray(headers[k], np.int64)
        hb = (np.asarray(h[0:7], e + "i4").tobytes() + np.asarray(h[7:11], e + "i2").tobytes()
              + np.asarray(h[11:19], e + "i4").tobytes() + np.asarray(h[19:21], e + "i2").tobytes()
              + np.asarray(h[21:25], e + "i4").tobytes() + np.asarray(h[25:101], e + "i2").tobytes())
        assert len(hb) == 240
        body.append(hb + np.asarray(samples[k], e + sdt).tobytes())
    with open(path, "wb") as f:
        f.write(tb + reel + b"".join(body))


def interp1_linear(traces: np.ndarray, levels: int) -> np.ndarray:
    """ktmInterpTraceBlock.m opt 2 in FP64, rounded to float32 at the end."""
    x = np.asarray(traces, np.float64)
    ntr, nt = x.shape
    if nt < 2:
        return x.astype(np.float32)
    nout = (nt - 1) * (1 << levels) + 1
    j = np.arange(nout)
    i = np.minimum(j >> levels, nt - 2)
    s = j / float(1 << levels) - i                  # t' - i, exact
    y = (x[:, i + 1] - x[:, i]) * s + x[:, i]
    return y.astype(np.float32)
