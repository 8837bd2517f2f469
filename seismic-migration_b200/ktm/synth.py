"""Seeded synthetic surveys for the tests and the benchmark.

No field data ships with the reference and none is available here, so the
workloads are synthetic, built the way the reference's impulse option builds
test data (scripts/ktmWriteTraceBlockConstOffset.m:65-83 spikes a zero block)
but with diffraction responses instead of bare spikes:

  * a line (2-D) survey: CMPs on x at 12.5 m, constant-offset bins, one trace
    per (offset bin, CMP), traces grouped by offset as the constant-offset
    writer groups them;
  * an areal (3-D) survey: sources and receivers uniform over a square,
    offsets up to a maximum with uniform azimuth;
  * traces = sum over point scatterers of a Ricker wavelet at the
    double-square-root time from the source to the scatterer to the receiver
    (with the RMS velocity at the scatterer), plus Gaussian noise.

Conventions follow the reference: the image Z axis is one-way time tau
(zero-offset traveltime 2*tau), offsets are half-offset vectors
(ktmConvertXYtoOffMid.m:12), velocities are RMS velocities per tau sample.

Noise is a counter-based hash (splitmix64 -> Box-Muller) of (seed, trace,
sample), so the numpy generator here and the device generator
(``ktmSynthesizeTraces``) produce the same noise.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from ._lib import ImageGrid


@dataclass
class Survey:
    name: str
    imageX: ImageGrid
    imageY: ImageGrid
    imageZ: ImageGrid
    dt: float                       # trace sample interval, s
    nt: int                         # samples per trace
    midX: np.ndarray
    midY: np.ndarray
    offX: np.ndarray                # half offsets
    offY: np.ndarray
    velocity: np.ndarray            # [Nz] or [Nx][Ny][Nz], m/s
    velocity1d: np.ndarray          # [Nz] lateral mean (reference-mode path)
    scat: np.ndarray                # [ns, 5]: x, y, tau0, v_rms, amplitude
    freq: float                     # Ricker peak frequency, Hz
    noise: float                    # Gaussian noise sigma
    aperture: float                 # metres on |mid - x|
    rho_opt: int                    # ktmApplyRhoFilter option (1 2D, 2 2.5D, 3 3D)
    seed: int
    meta: dict = field(default_factory=dict)

    @property
    def ntr(self) -> int:
        return int(self.midX.shape[0])

    @property
    def shape(self):
        return (self.imageX.imagePnts, self.imageY.imagePnts, self.imageZ.imagePnts)

    @property
    def pairs(self) -> int:
        """Raw (image point, trace) pairs of one full migration."""
        nx, ny, nz = self.shape
        return nx * ny * nz * self.ntr

    def subset(self, k0: int, k1: int) -> "Survey":
        s = Survey(**{**self.__dict__})
        s.midX, s.midY = self.midX[k0:k1], self.midY[k0:k1]
        s.offX, s.offY = self.offX[k0:k1], self.offY[k0:k1]
        s.meta = {**self.meta, "trace_offset": self.meta.get("trace_offset", 0) + k0}
        return s


# ------------------------------------------------------------------------------- noise ---
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def hash_noise(seed: int, k0: int, ntr: int, nt: int) -> np.ndarray:
    """N(0,1) per (trace k0+i, sample j): Box-Muller on the two 32-bit halves of
    splitmix64(seed * 2^48 + k * 2^22 + j)  (k < 2^26, j < 2^22)."""
    k = np.arange(k0, k0 + ntr, dtype=np.uint64)[:, None]
    j = np.arange(nt, dtype=np.uint64)[None, :]
    with np.errstate(over="ignore"):
        ctr = (np.uint64(seed) << np.uint64(48)) + k * np.uint64(1 << 22) + j
    h = _splitmix64(ctr)
    u1 = ((h >> np.uint64(32)).astype(np.float64) + 0.5) * (1.0 / 4294967296.0)
    u2 = ((h & np.uint64(0xFFFFFFFF)).astype(np.float64) + 0.5) * (1.0 / 4294967296.0)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def ricker(t: np.ndarray, f: float) -> np.ndarray:
    a = (np.pi * f * t) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


# ------------------------------------------------------------------------- geometries ---
def line_survey(ncmp=256, dcmp=12.5, noff=64, doff=50.0, nt=1001, dt=0.004, nz=None,
                dtau=None, nscat=20, freq=25.0, noise=0.05, aperture=2000.0, rho_opt=2,
                seed=1, name="line") -> Survey:
    """2-D line: ncmp CMPs x noff constant-offset bins (0, doff, ...), traces
    ordered offset-major (trace k = o*ncmp + i).  Vrms(t0) = 1500 + 0.5 t0[ms]."""
    rng = np.random.default_rng(seed)
    nz = nt if nz is None else nz
    dtau = dt / 2.0 if dtau is None else dtau
    cmp_x = dcmp * np.arange(ncmp)
    h = doff * np.arange(noff)
    midX = np.tile(cmp_x, noff).astype(np.float32)
    offX = np.repeat(h / 2.0, ncmp).astype(np.float32)
    zeros = np.zeros(ncmp * noff, np.float32)
    tau = dtau * np.arange(nz)
    vel = (1500.0 + 0.5 * (2.0 * tau * 1000.0)).astype(np.float32)
    xmax = cmp_x[-1]
    tmax = dt * (nt - 1)
    sx = rng.uniform(0.0, xmax, nscat)
    st = rng.uniform(0.05 * tmax / 2, 0.9 * min(tmax / 2, dtau * (nz - 1)), nscat)
    sv = 1500.0 + 0.5 * (2.0 * st * 1000.0)
    sa = rng.uniform(-1.0, 1.0, nscat)
    scat = np.stack([sx, np.zeros(nscat), st, sv, sa], axis=1)
    return Survey(name, ImageGrid(ncmp, dcmp, 0.0), ImageGrid(1, 1.0, 0.0),
                  ImageGrid(nz, dtau, 0.0), dt, nt, midX, zeros.copy(), offX, zeros.copy(),
                  vel, vel.copy(), scat, freq, noise, aperture, rho_opt, seed)


def smooth_field(n1: int, n2: int, d: float, corr: float, rng) -> np.ndarray:
    """Seeded smooth random field in [-1, 1] with correlation length ~corr."""
    from scipy.ndimage import gaussian_filter
    w = rng.standard_normal((n1, n2))
    p = gaussian_filter(w, sigma=corr / d / 2.0, mode="wrap")
    return p / np.max(np.abs(p))


def areal_survey(ntr=1_000_000, side=5000.0, maxoff=4000.0, nx=200, ny=200, dxy=25.0,
                 nt=1501, dt=0.002, nz=None, nscat=200, freq=30.0, noise=0.05,
                 aperture=3000.0, vtop=1500.0, vbot=4000.0, lateral=0.05, corr=1000.0,
                 rho_opt=3, seed=2, name="areal") -> Survey:
    """3-D: sources and receivers uniform over side x side, |r - s| <= maxoff
    (uniform offset magnitude, uniform azimuth; receivers outside the square are
    re-drawn).  Vrms(x, y, t0) = (vtop + (vbot - vtop) t0/tmax) (1 + lateral P(x, y))."""
    rng = np.random.default_rng(seed)
    nz = nt if nz is None else nz
    dtau = dt / 2.0
    s = rng.uniform(0.0, side, (ntr, 2))
    r = np.empty_like(s)
    todo = np.arange(ntr)
    while todo.size:
        hm = rng.uniform(0.0, maxoff, todo.size)
        az = rng.uniform(0.0, 2.0 * np.pi, todo.size)
        cand = s[todo] + np.stack([hm * np.cos(az), hm * np.sin(az)], axis=1)
        ok = np.all((cand >= 0.0) & (cand <= side), axis=1)
        r[todo[ok]] = cand[ok]
        todo = todo[~ok]
    mid = (s + r) / 2.0
    off = (r - s) / 2.0
    gx = ImageGrid(nx, dxy, dxy / 2.0)
    gy = ImageGrid(ny, dxy, dxy / 2.0)
    gz = ImageGrid(nz, dtau, 0.0)
    tau = dtau * np.arange(nz)
    tmax = 2.0 * tau[-1]
    v0 = vtop + (vbot - vtop) * (2.0 * tau) / tmax
    P = smooth_field(nx, ny, dxy, corr, rng)
    vel = (v0[None, None, :] * (1.0 + lateral * P[:, :, None])).astype(np.float32)
    sx = rng.uniform(0.0, side, nscat)
    sy = rng.uniform(0.0, side, nscat)
    st = rng.uniform(0.05 * tau[-1], 0.9 * tau[-1], nscat)
    ix = np.clip(((sx - gx.imageStart) / dxy).round().astype(int), 0, nx - 1)
    iy = np.clip(((sy - gy.imageStart) / dxy).round().astype(int), 0, ny - 1)
    sv = (vtop + (vbot - vtop) * (2.0 * st) / tmax) * (1.0 + lateral * P[ix, iy])
    sa = rng.uniform(-1.0, 1.0, nscat)
    scat = np.stack([sx, sy, st, sv, sa], axis=1)
    return Survey(name, gx, gy, gz, dt, nt, mid[:, 0].astype(np.float32),
                  mid[:, 1].astype(np.float32), off[:, 0].astype(np.float32),
                  off[:, 1].astype(np.float32), vel, vel.mean(axis=(0, 1)).astype(np.float32),
                  scat, freq, noise, aperture, rho_opt, seed)


def config1(seed=1) -> Survey:
    """2D PSTM: 256 CMPs @ 12.5 m x 64 offsets (0-3150 m), 1001 samples @ 4 ms,
    20 scatterers, 25 Hz, sigma 0.05, 256 x 1001 image, aperture 2 km."""
    return line_survey(seed=seed, name="2d-line-256cmp-64off-1001")


def config2(ntr=1_000_000, seed=2) -> Survey:
    """3D PSTM: 200 x 200 @ 25 m, 1501 t0 @ 2 ms, 1e6 traces, 5 x 5 km, offsets
    <= 4 km, Vrms 1500 -> 4000 m/s +-5 % lateral (1 km), 200 scatterers, 30 Hz,
    sigma 0.05, aperture 3 km."""
    return areal_survey(ntr=ntr, seed=seed, name="3d-200x200x1501-1e6tr")


def config4(seed=4) -> Survey:
    """Adjoint / LSM: 512 CMPs x 64 offsets x 1001 samples @ 4 ms."""
    return line_survey(ncmp=512, seed=seed, name="2d-line-512cmp-64off-1001")


# ---------------------------------------------------------------------------- traces ---
def synthesize_device(sv: Survey, k0: int = 0, k1: int | None = None, device="cuda",
                      coords=None, out=None, stream=None):
    """Device traces [k1-k0, nt] float32 from ktmSynthesizeTraces (same recipe
    and noise as ``synthesize``).  ``coords`` = (midX, midY, offX, offY) CUDA
    tensors of the whole survey, to avoid re-uploading them."""
    import ctypes as C

    import torch

    from ._lib import check, lib
    k1 = sv.ntr if k1 is None else k1
    n = k1 - k0
    if coords is None:
        coords = [torch.as_tensor(np.ascontiguousarray(a)).to(device)
                  for a in (sv.midX, sv.midY, sv.offX, sv.offY)]
    scat = torch.as_tensor(np.ascontiguousarray(sv.scat, dtype=np.float64)).to(device)
    if out is None:
        out = torch.empty((n, sv.nt), device=device, dtype=torch.float32)
    mx, my, ox, oy = (c[k0:k1] for c in coords)
    stream_h = None if stream is None else stream.cuda_stream
    check(lib().ktmSynthesizeTraces(
        int(n), int(sv.nt), float(sv.dt), mx.data_ptr(), my.data_ptr(), ox.data_ptr(),
        oy.data_ptr(), int(scat.shape[0]), scat.data_ptr(), float(sv.freq), float(sv.noise),
        C.c_ulonglong(int(sv.seed)), int(sv.meta.get("trace_offset", 0) + k0), out.data_ptr(),
        stream_h))
    torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
    return out


def synthesize(sv: Survey, k0: int = 0, k1: int | None = None, noise: bool = True) -> np.ndarray:
    """Numpy traces [k1-k0, nt] float32 (CPU; meant for small surveys)."""
    k1 = sv.ntr if k1 is None else k1
    n = k1 - k0
    mx, my = sv.midX[k0:k1].astype(np.float64), sv.midY[k0:k1].astype(np.float64)
    ox, oy = sv.offX[k0:k1].astype(np.float64), sv.offY[k0:k1].astype(np.float64)
    out = np.zeros((n, sv.nt), np.float64)
    half = int(np.ceil(1.5 / sv.freq / sv.dt)) + 1
    win = np.arange(-half, half + 1)
    rows = np.arange(n)[:, None]
    for x, y, t0, v, a in sv.scat:
        ts = np.sqrt(t0 * t0 + ((mx - ox - x) ** 2 + (my - oy - y) ** 2) / (v * v))
        tr = np.sqrt(t0 * t0 + ((mx + ox - x) ** 2 + (my + oy - y) ** 2) / (v * v))
        t = ts + tr
        j = np.floor(t / sv.dt).astype(np.int64)[:, None] + win[None, :]
        ok = (j >= 0) & (j < sv.nt)
        val = a * ricker(j * sv.dt - t[:, None], sv.freq)
        np.add.at(out, (np.broadcast_to(rows, j.shape)[ok], j[ok]), val[ok])
    if noise and sv.noise > 0:
        out += sv.noise * hash_noise(sv.seed, sv.meta.get("trace_offset", 0) + k0, n, sv.nt)
    return out.astype(np.float32)


def encode_ibm32(x) -> np.ndarray:
    """IEEE -> IBM System/360 single precision words (sign, base-16 exponent
    biased by 64, 24-bit fraction in [1/16, 1)), rounding the fraction to
    nearest: synthetic IBM data of the kind inputData.bin holds.  Values beyond
    the IBM range clamp to its largest / smallest exponent."""
    a64 = np.asarray(x, np.float64)
    out = np.zeros(a64.shape, np.uint32)
    a = np.abs(a64)
    nz = a > 0
    if not nz.any():
        return out
    v = a[nz]
    e = np.floor(np.log2(v) / 4.0).astype(np.int64) + 1          # v = f 16^e, f in [1/16, 1)
    f = v / np.power(16.0, e.astype(np.float64))
    lo = f < 1.0 / 16.0
    e[lo] -= 1
    f[lo] *= 16.0
    hi = f >= 1.0
    e[hi] += 1
    f[hi] /= 16.0
    frac = np.rint(f * float(1 << 24)).astype(np.int64)
    up = frac >= (1 << 24)                                           # rounded up to 1.0
    frac[up] = 1 << 20
    e[up] += 1
    e = np.clip(e + 64, 0, 127)
    sign = (a64[nz] < 0).astype(np.int64) << 31
    out[nz] = (sign | (e << 24) | frac).astype(np.uint32)
    return out
