"""The CPU oracle, pinned against the reference's own outputs (golden fixtures
made by tests/golden/make_golden.py from the unmodified psktmCPU.c and
ioFunctions.c) and against analytic known answers."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import rho
from conftest import GOLDEN_MIGRATIONS, golden_grids, load_golden


@pytest.mark.parametrize("name", GOLDEN_MIGRATIONS)
def test_ref32_restatement_matches_reference_golden(name):
    g = load_golden(name)
    gx, gy, gz = golden_grids(g)
    img = oracle.migrate_ref32(gx, gy, gz, float(g["dt"]), g["midX"], g["midY"], g["offX"],
                               g["offY"], g["traces"], g["velocity"])
    # bit-identical, not merely close
    assert img.shape == g["image"].shape
    assert np.array_equal(img.view(np.uint32), g["image"].view(np.uint32))


def test_golden_fixtures_not_trivial():
    for name in GOLDEN_MIGRATIONS:
        g = load_golden(name)
        assert np.count_nonzero(g["image"]) > 0, name


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_ref32_restatement_matches_reference_library_random(seed):
    rng = np.random.default_rng(seed)
    ntr, nt = 37, 91
    gx, gy, gz = oracle.grid(5, 33.0, -60.0), oracle.grid(3, 21.0, 10.0), oracle.grid(77, 0.0025, 0.0)
    mid = rng.uniform(-200, 200, (ntr, 2)).astype(np.float32)
    off = rng.uniform(-300, 300, (ntr, 2)).astype(np.float32)
    tr = rng.standard_normal((ntr, nt)).astype(np.float32)
    vel = rng.uniform(1500, 3500, 77).astype(np.float32)
    a = oracle.migrate_ref32(gx, gy, gz, 0.004, mid[:, 0], mid[:, 1], off[:, 0], off[:, 1], tr, vel)
    b = oracle.migrate_reference_c(gx, gy, gz, 0.004, mid[:, 0], mid[:, 1], off[:, 0], off[:, 1],
                                   tr, vel, threads=1)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_f64_truncate_agrees_with_ref32():
    g = load_golden("ref_line_small.npz")
    gx, gy, gz = golden_grids(g)
    args = (gx, gy, gz, float(g["dt"]), g["midX"], g["midY"], g["offX"], g["offY"], g["traces"],
            g["velocity"])
    f64 = oracle.migrate_f64(*args, pick=0)
    ref = g["image"].astype(np.float64)
    # the FP32 reference can flip a truncated sample index where t/dt is within
    # an ulp of an integer; those are rare
    rel = np.linalg.norm(f64 - ref) / np.linalg.norm(ref)
    assert rel < 2e-3


def test_f64_linear_equals_truncate_on_integer_times():
    """One zero-offset trace under a one-column image, tau and dt powers of two:
    t/dt = 2 tau/dt is an exact integer, so linear interpolation reduces to the
    reference pick."""
    rng = np.random.default_rng(9)
    nt, nz = 64, 40
    gx, gy, gz = oracle.grid(1, 1.0, 10.0), oracle.grid(1, 1.0, 0.0), oracle.grid(nz, 2.0**-9, 0.0)
    tr = rng.standard_normal((1, nt)).astype(np.float32)
    one = np.array([10.0], np.float32)
    z = np.zeros(1, np.float32)
    args = (gx, gy, gz, 2.0**-8, one, z, z, z, tr, np.full(nz, 1800.0, np.float32))
    a = oracle.migrate_f64(*args, pick=0)
    b = oracle.migrate_f64(*args, pick=1)
    assert np.count_nonzero(a) > nz // 2
    assert np.allclose(a, b, rtol=1e-12, atol=1e-12)


def test_f64_column_subset():
    g = load_golden("ref_areal_small.npz")
    gx, gy, gz = golden_grids(g)
    args = (gx, gy, gz, float(g["dt"]), g["midX"], g["midY"], g["offX"], g["offY"], g["traces"],
            g["velocity"])
    full = oracle.migrate_f64(*args, aperture=250.0)
    sub = oracle.migrate_f64(*args, aperture=250.0, columns=(7, 9))
    assert np.array_equal(full.reshape(-1, gz.imagePnts)[7:16], sub)


def test_f64_adjoint_dot_product():
    rng = np.random.default_rng(5)
    ntr, nt = 23, 120
    gx, gy, gz = oracle.grid(6, 25.0, 0.0), oracle.grid(2, 25.0, 0.0), oracle.grid(60, 0.002, 0.0)
    mid = rng.uniform(0, 150, (ntr, 2)).astype(np.float32)
    off = rng.uniform(-100, 100, (ntr, 2)).astype(np.float32)
    vel = np.linspace(1500, 2500, 60).astype(np.float32)
    d = rng.standard_normal((ntr, nt)).astype(np.float32)
    m = rng.standard_normal((6, 2, 60))
    for pick, prefold in ((0, 0), (1, 0), (1, 1), (1, 3)):
        Ld = oracle.migrate_f64(gx, gy, gz, 0.004, mid[:, 0], mid[:, 1], off[:, 0], off[:, 1], d,
                                vel, pick=pick, aperture=120.0, prefold=prefold)
        Ltm = oracle.demigrate_f64(gx, gy, gz, 0.004, mid[:, 0], mid[:, 1], off[:, 0], off[:, 1], nt,
                                   vel, m, pick=pick, aperture=120.0, prefold=prefold)
        lhs, rhs = np.vdot(Ld, m), np.vdot(d.astype(np.float64), Ltm)
        assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


def test_ibm32_restatement_matches_reference_golden():
    g = load_golden("ref_ibm32.npz")
    out = oracle.ibm32_to_ieee(g["words"])
    assert np.array_equal(out.view(np.uint32), g["ieee"].view(np.uint32))


def test_ibm32_known_values():
    # IBM 0x41100000 = +1.0 * 16^1 * (0x100000 / 0xFFFFFF) (the reference divides by
    # FRACTION_MASK, ioFunctions.c:33, not by 2^24)
    out = oracle.ibm32_to_ieee(np.array([0x41100000, 0xC2640000, 0x00000000], np.uint32))
    assert out[0] == np.float32(np.float32(0x100000) / np.float32(0xFFFFFF)) * np.float32(16.0)
    assert out[1] < 0 and abs(out[1] + 100.0) < 1e-3
    assert out[2] == 0.0


# --------------------------------------------------------------------------- rho filter ---
@pytest.mark.parametrize("opt", [1, 2, 3])
def test_rho_known_answer_single_tone(opt):
    """A tone on an exact FFT bin k0 (m = M = 256, so no padding): the filter
    multiplies it by |H(2 pi k0 / Dr)|, shifts its phase by arg H.  No 1/M in
    omega: the reference's scaling (ktmApplyRhoFilter.m:33)."""
    M, k0, dw = 256, 9, 4000.0
    n = np.arange(M)
    x = np.cos(2 * np.pi * k0 * n / M)
    w = 2 * np.pi * k0 / (dw * 1e-6)
    if opt == 1:
        expect = w * x
    elif opt == 2:
        expect = np.sqrt(w) * np.cos(2 * np.pi * k0 * n / M + np.pi / 4)
    else:
        expect = -w * np.sin(2 * np.pi * k0 * n / M)
    got = rho.apply_rho_filter(x[None, :], dw, opt)[0]
    assert np.allclose(got, expect, rtol=1e-9, atol=1e-9 * np.abs(expect).max())


def test_rho_padding_and_truncation():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((4, 1001))
    assert rho.fft_length(1001) == 1024 and rho.fft_length(1501) == 2048
    y = rho.apply_rho_filter(x, 4000.0, 2)
    assert y.shape == x.shape
    # linear in the traces
    y2 = rho.apply_rho_filter(2.0 * x, 4000.0, 2)
    assert np.allclose(y2, 2.0 * y)


def test_rho_octave_matrix_fftshift_rotates_odd_trace_counts():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((5, 100))
    per_trace = rho.rho_filter_traces(x, 2000.0, 3)
    script = rho.apply_rho_filter(x, 2000.0, 3)
    assert np.allclose(script, np.roll(per_trace, -1, axis=0))
    x = x[:4]
    assert np.allclose(rho.apply_rho_filter(x, 2000.0, 3), rho.rho_filter_traces(x, 2000.0, 3))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
def test_ref32_restatement_matches_reference_library_degenerate():
    """Zero, negative, huge, infinite and NaN velocities and infinite trace samples:
    the restatement reproduces the reference's NaN and infinite image samples."""
    from conftest import degenerate_reference_case, same_with_nans
    args = degenerate_reference_case()
    a = oracle.migrate_ref32(*args)
    b = oracle.migrate_reference_c(*args, threads=1)
    assert np.isnan(b).any() and np.isinf(b).any() and np.isfinite(b).any()
    assert same_with_nans(a, b)
