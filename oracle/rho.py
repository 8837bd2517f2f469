"""NumPy FP64 restatement of the rho (half-derivative) pre-filter.
TEST INFRASTRUCTURE ONLY (the checker for the device rho-filter kernel).

Follows scripts/ktmApplyRhoFilter.m:22-62 line by line:
  * input ``trace`` is [n traces, m samples] (rows are traces, :22);
  * FFT length M = 2^ceil(log2 m), zero padding (:26, :37);
  * Dr = dw * 1e-6 (dw is the sample interval in microseconds, :31);
  * omega = 2*pi*(-M/2 .. M/2-1) / Dr, paired with the fftshift-ed spectrum
    (:33, :37) -- note there is no 1/M, so the filter is M times a true
    derivative operator; this is the reference's scaling and is kept;
  * opt 1 (2D): |omega|; opt 2 (2.5D): sqrt|omega| * exp(i*pi/4*sign(omega));
    anything else (3D): i*omega  (:39-58);
  * output real(ifft(fftshift(H .* F))) truncated to the first m samples.
  * Octave's fftshift of a MATRIX shifts every dimension, so the two calls at
    :37 and :43/:50/:57 also rotate the trace (column) axis twice by
    ceil(n/2): for an odd trace count n > 1 output trace q is the filtered
    input trace (q+1) mod n.  ``apply_rho_filter`` keeps this;
    ``rho_filter_traces`` is the per-trace filter without the rotation.

Octave is not installed, so this restatement cannot be run against the
script itself; it is pinned by analytic known answers (tests/test_oracle.py).
"""
from __future__ import annotations

import numpy as np


def fft_length(m: int) -> int:
    """M = 2^ceil(log(m)/log(2)) (ktmApplyRhoFilter.m:26)."""
    return 1 << int(np.ceil(np.log2(m))) if m > 1 else 1


def rho_response(M: int, dw_us: float, opt: int) -> np.ndarray:
    """Filter sampled on the fftshift-ed frequency grid (index j <-> k = j - M/2)."""
    dr = dw_us * 1e-6
    omega = 2.0 * np.pi * (np.arange(M) - M // 2) / dr
    if opt == 1:
        return np.abs(omega).astype(np.complex128)
    if opt == 2:
        return np.sqrt(np.abs(omega)) * np.exp((1j * np.pi / 4.0) * np.sign(omega))
    return 1j * omega


def _octave_fftshift(x: np.ndarray) -> np.ndarray:
    """Octave fftshift: a vector shifts along its length, a matrix along every
    dimension, each by ceil(L/2) (x(idx) with idx = [ceil(L/2)+1:L, 1:ceil(L/2)])."""
    if x.ndim == 2 and 1 in x.shape:
        return np.roll(x, -((max(x.shape) + 1) // 2), axis=0 if x.shape[1] == 1 else 1)
    for ax in range(x.ndim):
        x = np.roll(x, -((x.shape[ax] + 1) // 2), axis=ax)
    return x


def rho_filter_traces(trace: np.ndarray, dw_us: float, opt: int) -> np.ndarray:
    """Per-trace rho filter (each row filtered on its own)."""
    trace = np.atleast_2d(np.asarray(trace, dtype=np.float64))
    n, m = trace.shape
    M = fft_length(m)
    F = np.fft.fftshift(np.fft.fft(trace, M, axis=1), axes=1)
    H = rho_response(M, dw_us, opt)[None, :]
    out = np.real(np.fft.ifft(np.fft.ifftshift(H * F, axes=1), axis=1))
    return out[:, :m]


def apply_rho_filter(trace: np.ndarray, dw_us: float, opt: int) -> np.ndarray:
    """ktmApplyRhoFilter(trace, dw, opt) as the script computes it."""
    trace = np.atleast_2d(np.asarray(trace, dtype=np.float64))
    n, m = trace.shape
    M = fft_length(m)
    F = _octave_fftshift(np.fft.fft(trace.T, M, axis=0))             # :37 (M x n)
    H = np.repeat(rho_response(M, dw_us, opt)[:, None], n, axis=1)   # :33 repmat
    out = np.real(np.fft.ifft(_octave_fftshift(H * F), axis=0)).T    # :43/:50/:57
    return out[:, :m]
