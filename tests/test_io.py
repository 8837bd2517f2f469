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


# ---- the reference's file functions under their own names (ioFunctions.c:44-153) ----

def _libs():
    import ctypes as C

    import oracle
    from conftest import PKG  # noqa: F401
    import ktm
    libc = C.CDLL("libc.so.6")
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    libc.ftell.restype = C.c_long
    libc.ftell.argtypes = [C.c_void_p]
    libc.fread.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p]
    libc.fread.restype = C.c_size_t
    libc.free.argtypes = [C.c_void_p]
    libs = [ktm.lib()]
    if oracle.ref_available():
        libs.append(C.CDLL(oracle.REF_SO))
    for L in libs:
        L.fileSizeFourBytes.argtypes = [C.c_void_p]
        L.fileSizeFourBytes.restype = C.c_int
        for fn in ("binReadUints", "binReadFloats"):
            getattr(L, fn).argtypes = [C.c_void_p, C.c_int]
            getattr(L, fn).restype = C.c_void_p
        L.fileWrite.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.fileWrite.restype = None
        L.loadInputData.argtypes = [C.c_void_p]
        L.loadInputData.restype = None
    return libc, libs


class _FileInputPtrs(__import__("ctypes").Structure):
    import ctypes as _C
    _fields_ = [("flag", _C.c_int), ("inputData", _C.c_void_p), ("inputSrcX", _C.c_void_p),
                ("inputSrcY", _C.c_void_p), ("inputRecX", _C.c_void_p), ("inputRecY", _C.c_void_p)]


def test_reference_file_functions_match_ioFunctions(tmp_path):
    """fileSizeFourBytes / binReadUints / binReadFloats / fileWrite of the library
    against the reference's own compiled ioFunctions.c: same counts, words and
    bytes, and the file left at its start."""
    import ctypes as C
    libc, libs = _libs()
    words = np.random.default_rng(3).integers(0, 2**32, 1001, dtype=np.uint64).astype(np.uint32)
    path = tmp_path / "w.bin"
    path.write_bytes(words.tobytes() + b"\x01\x02\x03")          # 3 stray bytes at the end
    results = []
    for k, L in enumerate(libs):
        f = libc.fopen(str(path).encode(), b"rb")
        n = L.fileSizeFourBytes(f)
        pos = libc.ftell(f)
        pu = L.binReadUints(f, n)
        u = np.ctypeslib.as_array(C.cast(pu, C.POINTER(C.c_uint32)), (n,)).copy()
        pf = L.binReadFloats(f, 10)
        fl = np.ctypeslib.as_array(C.cast(pf, C.POINTER(C.c_float)), (10,)).copy()
        pos2 = libc.ftell(f)
        libc.free(pu)
        libc.free(pf)
        libc.fclose(f)
        out = tmp_path / f"out{k}.bin"
        g = libc.fopen(str(out).encode(), b"wb")
        vals = np.linspace(-1.0, 1.0, 77).astype(np.float32)
        L.fileWrite(g, vals.ctypes.data, 77)
        libc.fclose(g)
        results.append((n, pos, u, fl, pos2, out.read_bytes()))
    n, pos, u, fl, pos2, wrote = results[0]
    assert n == 1001 and pos == 0 and pos2 == 0
    assert np.array_equal(u, words)
    assert np.array_equal(fl.view(np.uint32), words[:10])
    assert wrote == np.linspace(-1.0, 1.0, 77).astype(np.float32).tobytes()
    for other in results[1:]:                     # the reference's compiled code
        assert other[0] == n and other[1] == pos and other[4] == pos2
        assert np.array_equal(other[2], u) and np.array_equal(other[3].view(np.uint32), fl.view(np.uint32))
        assert other[5] == wrote


def test_reference_load_input_data(tmp_path):
    """loadInputData opens ../data/*.bin relative to the working directory, as the
    reference does; a missing file sets flag = 1 and prints the reference's message.
    Run in a child process so that the working directory and stdout are its own."""
    import subprocess
    import sys
    data = tmp_path / "data"
    work = tmp_path / "work"
    data.mkdir()
    work.mkdir()
    for i, name in enumerate(("inputData", "inputSrcX", "inputSrcY", "inputRecX", "inputRecY")):
        (data / f"{name}.bin").write_bytes(np.arange(i, i + 8, dtype=np.float32).tobytes())
    prog = r'''
import ctypes as C, sys
sys.path[:0] = sys.argv[1].split(":")
import test_io
libc, libs = test_io._libs()
for L in libs:
    s = test_io._FileInputPtrs()
    L.loadInputData(C.byref(s))
    firsts = []
    for fld in ("inputData", "inputSrcX", "inputSrcY", "inputRecX", "inputRecY"):
        f = getattr(s, fld)
        v = C.c_float()
        libc.fread(C.byref(v), 4, 1, f) if f else None
        firsts.append(v.value if f else None)
    print("RESULT", s.flag, firsts, flush=True)
'''
    here = os.path.dirname(os.path.abspath(__file__))
    pp = ":".join([here, os.path.join(os.path.dirname(here), "seismic-migration_b200"),
                   os.path.join(os.path.dirname(here), "oracle")])
    out = subprocess.run([sys.executable, "-c", prog, pp], cwd=work, capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    res = [ln for ln in out.stdout.splitlines() if ln.startswith("RESULT")]
    assert res and all(r == "RESULT 0 [0.0, 1.0, 2.0, 3.0, 4.0]" for r in res), out.stdout
    (data / "inputRecX.bin").unlink()
    out = subprocess.run([sys.executable, "-c", prog, pp], cwd=work, capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    res = [ln for ln in out.stdout.splitlines() if ln.startswith("RESULT")]
    assert res and all(r.startswith("RESULT 1 [0.0, 1.0, 2.0, None, 4.0]") for r in res), out.stdout
    assert out.stdout.count("Can't open ../data/inputRecX.bin.") == len(res)
