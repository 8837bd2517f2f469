"""Benchmark: 3-D prestack Kirchhoff time migration on B200.

Workload (one GPU): a 200 x 200 x 1501 image (25 m bins, t0 at 2 ms, so tau at
1 ms one-way) from 1,000,000 traces of 1501 samples at 2 ms; sources and
receivers uniform over 5 x 5 km, offsets <= 4 km, uniform azimuth; Vrms
1500 -> 4000 m/s with a seeded +-5 % lateral field (1 km correlation);
traces = 30 Hz Ricker diffractions from 200 scatterers plus sigma 0.05 noise
(seeded, synthesised on the device); aperture 3 km.  No public dataset exists
for this path, so the data are synthetic with the stated shapes.

A step = one batch of traces (1/16 of the survey by default) through the hot
path: the rho pre-filter (3-D, i*omega) and FP16 packing with a per-trace
scale (ktmPrepareTraces), then the mixed-precision
gather kernel accumulating into the resident image (ktmMigrate).  16 steps =
the whole job.  Each batch's traces (375 MB) exceed the 126 MB L2.

Printed: one JSON line.  ``value`` = raw image-point x trace pairs per second
of the mixed path with inputs resident in HBM; ``e2e`` = the same through the
C ABI with host buffers (host->device copies and the image read-back inside
the timed region); ``plain_fp32`` = the bit-exact FP32 kernel (psktmCPU.c
arithmetic) on the same geometry; ``error`` = relative L2 / max error of one
batch's image against the FP64 device evaluation on sampled columns;
``cpu_baseline`` = the reference's own psktmCPU.c on this host's cores.

``--impl reference`` runs the reference's CPU implementation instead
(oracle/_ref, built from the reference sources; rank 0 only).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "seismic-migration_b200"))

METRIC = "PSTM G(image-pt x trace)/s on 1 B200: mixed vs plain FP32 @<=1e-3 rel L2 err"
UNIT = "Gpair/s"
WORKLOAD = "3D PSTM 200x200x1501 image, 1e6 traces x 1501 samples @ 2 ms, aperture 3 km"

# DRAM read + write of the migration kernel per trace of a step on the full 200 x 200 x
# 1501 image (FP16 packed traces, five launches of 40 MB trace blocks per 62,500-trace
# step): 3.76 GB per step from one ncu capture of a full bench step
# (profiles/migrate_fast_3d-62500-traces_dram-traffic.md), divided by its traces.
MIGRATE_DRAM_BYTES_PER_TRACE = 3.76e9 / 62500
MIGRATE_DRAM_NOTE = ("DRAM read+write per step from one ncu capture of a full step (5 launches "
                     "of the kernel, one per 40 MB trace block), scaled by the traces of the "
                     "step; measured on the whole image (N=1)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ntr", type=int, default=1_000_000)
    ap.add_argument("--batches", type=int, default=16)
    ap.add_argument("--fmt", default="f16", choices=["f16", "bf16", "f32"])
    ap.add_argument("--err-side", type=int, default=64,
                    help="error check on a seeded random SIDE x SIDE x Nz subgrid (FP64 device)")
    ap.add_argument("--e2e-steps", type=int, default=None,
                    help="steps of the end-to-end measurement (default: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-plain", action="store_true", help="skip the plain FP32 comparison")
    ap.add_argument("--skip-error", action="store_true", help="skip the FP64 error check")
    ap.add_argument("--config", default="3d", choices=["3d", "batch", "2d", "lsm"],
                    help="3d: the headline workload; batch: 64 target-oriented jobs in one "
                         "persistent launch")
    ap.add_argument("--jobs", type=int, default=64)
    ap.add_argument("--lsm-jobs", type=int, default=None,
                    help="--config batch: jobs that run 10 CGLS iterations (default: all)")
    ap.add_argument("--batch-fmt", default="both", choices=["f16", "bf16", "both"],
                    help="--config batch: trace formats to time (both: FP16 first, BF16 beside)")
    ap.add_argument("--err-cols", type=int, default=64,
                    help="--config batch: sampled columns per job for the error")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-step-seconds", type=float, default=None,
                    help="--impl reference: CPU seconds per step (default: about 150 s "
                         "spread over warm-up and timed steps, at least 2 s each)")
    ap.add_argument("--tile-run", type=int, default=0,
                    help="tau samples per warp run: 256, 384 or 512 (0: chosen by Nz)")
    ap.add_argument("--weight", default="prefold", choices=["prefold", "table", "sqrt"],
                    help="sqrt(t) of the weight: folded into the packed samples as sqrt(j dt) "
                         "(default), from the kernel's interpolated sqrt(j dt) table, or one "
                         "sqrt.approx per pair")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------
class CpuReference:
    """The reference's psktmCPU.c (oracle/_ref, compiled unmodified) or, where it
    was never built, the oracle's single-thread restatement, on a bounded sample
    of the workload: the full image against the first T traces.

    psktmCPU.c spreads its trace loop over the OpenMP threads (psktmCPU.c:56-59),
    so T is sized from a probe that gives every thread two traces, then rounded
    up to a multiple of the thread count with at least eight traces per thread,
    so that no thread idles in a last partial wave."""

    def __init__(self, sv, seconds: float, threads: int):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        self.oracle = oracle
        self.kind = "reference" if oracle.ref_available() else "port"
        self.threads = threads if self.kind == "reference" else 1
        g = oracle.grid
        self.grids = tuple(g(x.imagePnts, x.imageStep, x.imageStart)
                           for x in (sv.imageX, sv.imageY, sv.imageZ))
        self.sv = sv
        self.npts = int(np.prod(sv.shape))
        self.tr = np.random.default_rng(5).standard_normal((sv.ntr, sv.nt)).astype(np.float32)
        th = self.threads
        probe = min(sv.ntr, 2 * th)
        rate = probe / self.run(probe)                     # traces per second, all threads
        t = int(seconds * rate)
        t = max(t, 8 * th)
        t = -(-t // th) * th                               # whole waves of the thread team
        self.ntr = max(1, min(sv.ntr, t))

    def run(self, ntr: int) -> float:
        sv = self.sv
        args = (*self.grids, sv.dt, sv.midX[:ntr], sv.midY[:ntr], sv.offX[:ntr],
                sv.offY[:ntr], self.tr[:ntr], sv.velocity1d)
        t0 = time.perf_counter()
        if self.kind == "reference":
            self.oracle.migrate_reference_c(*args, threads=self.threads)
        else:
            self.oracle.migrate_ref32(*args)
        return time.perf_counter() - t0

    def rate(self) -> float:
        """pairs/s of one timed run of the sized sample."""
        return self.npts * self.ntr / self.run(self.ntr)

    def sample(self) -> str:
        nx, ny, nz = self.sv.shape
        pairs = self.npts * self.ntr
        if self.kind == "reference":
            return (f"full {nx}x{ny}x{nz} image x first {self.ntr} traces ({pairs:.3e} pairs, "
                    f"{self.ntr // self.threads} per thread), 1-D RMS velocity, "
                    f"{self.threads} OpenMP threads")
        return f"full image x first {self.ntr} traces, single-thread oracle restatement"


def cpu_reference_rate(sv, seconds: float, threads: int):
    """(pairs/s, cores, kind, sample) of the reference CPU code on a sized sample."""
    ref = CpuReference(sv, seconds, threads)
    return ref.rate(), ref.threads, ref.kind, ref.sample()


def reference_arm(a):
    """--impl reference: the reference's CPU implementation of the path, rank 0."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from ktm import synth
    sv = synth.config2(ntr=20000)
    threads = os.cpu_count() or 1
    budget = (a.ref_step_seconds if a.ref_step_seconds is not None
              else max(2.0, 150.0 / max(1, a.steps + a.warmup)))
    ref = CpuReference(sv, budget, threads)
    rates = []
    for i in range(a.warmup + a.steps):
        r = ref.rate()
        if i >= a.warmup:
            rates.append(r)
    v = float(np.mean(rates)) / 1e9
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "per_step": "bounded CPU sample, see cpu_baseline"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": ref.threads, "kind": ref.kind,
                         "sample": ref.sample()},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def rho_filter_f64(traces, dt: float, opt: int):
    """FP64 rho filter of ktmApplyRhoFilter.m:22-62, trace by trace, on the traces'
    device: zero padding to M = 2^ceil(log2 m), omega_k = 2 pi k / dt for the FFT's
    k = -M/2 .. M/2-1 (the script's scaling, no 1/M), 2D |omega|, 2.5D
    sqrt|omega| exp(i pi/4 sign omega), 3D i omega; the real part of the inverse
    FFT, truncated to m samples.  The first stage of the FP64 pipeline the bench's
    image error is measured against; returns float64 [n, m]."""
    import math

    import torch
    x = traces.double()
    m = x.shape[1]
    M = 1 << (m - 1).bit_length() if m > 1 else 1
    F = torch.fft.fft(x, n=M, dim=1)
    k = torch.fft.fftfreq(M, d=1.0 / M, device=x.device, dtype=torch.float64)
    omega = 2.0 * math.pi * k / float(dt)
    if opt == 1:
        H = omega.abs().to(torch.complex128)
    elif opt == 2:
        H = omega.abs().sqrt() * torch.exp(1j * (math.pi / 4.0) * torch.sign(omega))
    else:
        H = 1j * omega
    return torch.fft.ifft(F * H[None, :], dim=1).real[:, :m].contiguous()


# ---------------------------------------------------------------------------------------
def batch_main(a):
    """64 target-oriented jobs in ONE persistent launch (ktmMigrateBatch).

    Patch sides log-uniform in [16, 128] bins of 12.5 m, 751 tau samples (t0 at
    4 ms); trace counts log-uniform in [1e4, 5e5]; per job, sources and receivers
    uniform over the patch grown by the 2 km aperture, offsets <= 3150 m, the
    line survey's Vrms(t0) = 1500 + 0.5 t0[ms], 25 Hz Ricker diffractions from
    20 scatterers plus sigma 0.05 noise, 2.5-D rho filter, sqrt(j dt) folded in,
    a per-trace FP32 scale, FP32 accumulation, tile shape from ktmAutotune.

    Each trace format (FP16 by default, BF16 beside it) is timed as one launch over
    all jobs; every job's error is measured against an FP64 pipeline from its raw
    traces (FP64 rho filter, FP64 migration) on sampled columns; then 10 CGLS
    iterations (one iteration captured in a CUDA graph and replayed) per job."""
    import torch

    import ktm
    from ktm import synth
    from ktm.inverse import MigrationOperator
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(55)
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x, dtype=np.float32)).to(dev)  # noqa: E731
    fmts = ["f16", "bf16"] if a.batch_fmt == "both" else [a.batch_fmt]
    geos, packs, surveys = [], {f: [] for f in fmts}, []
    t0 = time.perf_counter()
    for j in range(a.jobs):
        side = int(round(np.exp(rng.uniform(np.log(16), np.log(128)))))
        ntr = int(round(np.exp(rng.uniform(np.log(1e4), np.log(5e5)))))
        box = side * 12.5 + 2 * 2000.0
        sv = synth.areal_survey(ntr=ntr, side=box, maxoff=3150.0, nx=side, ny=side, dxy=12.5,
                                nt=751, dt=0.004, nz=751, nscat=20, freq=25.0, noise=0.05,
                                aperture=2000.0, vtop=1500.0, vbot=1500.0 + 0.5 * 3000.0,
                                lateral=0.0, rho_opt=2, seed=1000 + j, name=f"job{j}")
        # the patch sits in the middle of its box
        sv.imageX.imageStart = sv.imageY.imageStart = 2000.0 + 6.25
        coords = [T(x) for x in (sv.midX, sv.midY, sv.offX, sv.offY)]
        raw = synth.synthesize_device(sv, device=dev, coords=coords)
        for f in fmts:
            packs[f].append(ktm.prepare(raw, sv.dt, fmt=f, rho=sv.rho_opt, prefold=True))
        del raw
        geos.append(dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt,
                         midX=coords[0], midY=coords[1], offX=coords[2], offY=coords[3],
                         velocity=T(sv.velocity1d), pick="linear", aperture=sv.aperture))
        surveys.append(sv)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    pairs = sum(s.pairs for s in surveys)
    runs, images = {}, {}
    for f in fmts:
        imgs = [torch.empty(s.shape, device=dev, dtype=torch.float32) for s in surveys]
        jobs = [dict(g, traces=p, image=im) for g, p, im in zip(geos, packs[f], imgs)]
        tune = ktm.autotune_tile(**jobs[int(np.argmax([s.pairs for s in surveys]))])
        for kw in jobs:
            kw["tile"] = tune
        ktm.migrate_batch(jobs)                               # warm-up
        torch.cuda.synchronize()
        times = []
        for _ in range(max(1, a.steps)):
            e0, e1 = _events()
            e0.record()
            ktm.migrate_batch(jobs)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = float(np.median(times))
        runs[f] = {"value": pairs / (ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_launch": ms,
                   "launches": len(times), "tile": tune}
        images[f] = imgs
    # every job's error against the FP64 pipeline from its raw traces, on sampled columns
    per_job = []
    for j, (sv, g) in enumerate(zip(surveys, geos)):
        raw = synth.synthesize_device(sv, device=dev, coords=[g[k] for k in ("midX", "midY", "offX", "offY")])
        nx, ny, nz = sv.shape
        cols = torch.as_tensor(np.sort(rng.choice(nx * ny, size=min(a.err_cols, nx * ny),
                                                  replace=False)).astype(np.int32))
        f64 = rho_filter_f64(raw, sv.dt, sv.rho_opt)
        ref = ktm.migrate_columns_f64(columns=cols, traces=f64, **g).double()
        del f64, raw
        row = {"job": j, "side": nx, "traces": sv.ntr, "columns": int(cols.numel())}
        for f in fmts:
            got = images[f][j].reshape(nx * ny, nz)[cols.to(dev).long()].double()
            row[f] = float((got - ref).norm() / ref.norm())
        per_job.append(row)
    errors = {}
    for f in fmts:
        e = np.array([r[f] for r in per_job])
        errors[f] = {"max": float(e.max()), "median": float(np.median(e)), "jobs": len(e),
                     "over_1e-3": int((e > 1e-3).sum())}
    # 10-iteration CGLS per job (one iteration graph-captured), on the job's rho-filtered data,
    # with the prefolded operator pair (the same weight as the batched migration)
    lsm = []
    nlsm = len(surveys) if a.lsm_jobs is None else min(a.lsm_jobs, len(surveys))
    order = np.argsort([s.pairs for s in surveys])[:nlsm]
    t_all = time.perf_counter()
    for j in sorted(order):
        sv, g = surveys[j], geos[j]
        op = MigrationOperator(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt,
                               nt=sv.nt, midX=g["midX"], midY=g["midY"], offX=g["offX"],
                               offY=g["offY"], velocity=g["velocity"], aperture=sv.aperture,
                               weight="prefold")
        raw = synth.synthesize_device(sv, device=dev, coords=[g[k] for k in ("midX", "midY", "offX", "offY")])
        d = op.pack(ktm.prepare(raw, sv.dt, fmt="f32", rho=sv.rho_opt, prefold=False).unpacked())
        del raw
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        _, rn, _ = op.least_squares(d, 10, use_graph=True)
        lsm.append({"job": int(j), "traces": sv.ntr, "side": sv.shape[0],
                    "residual_ratio": float(rn[-1] / rn[0]), "seconds": time.perf_counter() - t1})
        del d
    lsm_s = time.perf_counter() - t_all
    main_fmt = fmts[0]
    print(json.dumps({
        "metric": METRIC, "config": {"workload": f"batched: {len(surveys)} jobs in one persistent launch",
                                     "patch_sides": [s.shape[0] for s in surveys],
                                     "traces": [s.ntr for s in surveys], "nz": 751,
                                     "trace_format": main_fmt,
                                     "weight": "sqrt(j dt) folded into the packed samples"},
        "value": runs[main_fmt]["value"], "unit": UNIT, "pairs": pairs, "formats": runs,
        "error_rel_l2": errors,
        "error_vs": ("FP64 pipeline from each job's raw traces: FP64 rho filter (2.5-D), then FP64 "
                     f"migration (|tau| sqrt(t) per pair); {a.err_cols} sampled columns per job"),
        "per_job": per_job,
        "lsm_10_iterations": {"jobs": len(lsm), "seconds_total": lsm_s,
                              "residual_ratio_max": max((r["residual_ratio"] for r in lsm), default=None),
                              "per_job": lsm},
        "setup_s": setup_s,
    }), flush=True)


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def line_main(a):
    """The 2-D line (256 CMPs x 64 offsets, 16,384 traces of 1001 samples at 4 ms,
    256 x 1001 image, aperture 2 km, 2.5-D rho filter) in FP32, FP16 and BF16 with a
    per-trace FP32 scale (prefolded weight): throughput of each, its relative L2 and
    max error against the FP64 device evaluation of the WHOLE image, the plain FP32
    (bit-exact psktmCPU.c arithmetic) kernel on the same traces, and the reference's
    own psktmCPU.c on all host threads over the whole job."""
    import torch

    import ktm
    from ktm import synth
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    sv = synth.config1()
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x, dtype=np.float32)).to(dev)  # noqa: E731
    coords = [T(x) for x in (sv.midX, sv.midY, sv.offX, sv.offY)]
    raw = synth.synthesize_device(sv, device=dev, coords=coords)
    vel = T(sv.velocity1d)
    nx, ny, nz = sv.shape
    npts = nx * ny * nz
    geo = dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt, midX=coords[0],
               midY=coords[1], offX=coords[2], offY=coords[3], velocity=vel,
               aperture=sv.aperture)
    p32 = ktm.prepare(raw, sv.dt, fmt="f32", rho=sv.rho_opt, prefold=False)
    ref = ktm.migrate_columns_f64(ncols=nx * ny, traces=p32, pick="linear", **geo).double()
    out = {}
    for fmt in ("f32", "f16", "bf16"):
        p = ktm.prepare(raw, sv.dt, fmt=fmt, rho=sv.rho_opt, prefold=True)
        img = torch.empty(sv.shape, device=dev, dtype=torch.float32)
        for _ in range(max(3, a.warmup)):
            ktm.migrate(traces=p, image=img, pick="linear", **geo)
        e0, e1 = _events()
        e0.record()
        for _ in range(a.steps):
            ktm.migrate(traces=p, image=img, pick="linear", **geo)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.steps
        got = img.reshape(nx * ny, nz).double()
        out[fmt] = {"gpair_s": npts * sv.ntr / (ms * 1e-3) / 1e9, "ms": ms,
                    "rel_l2": float((got - ref).norm() / ref.norm()),
                    "max_rel": float((got - ref).abs().max() / ref.abs().max())}
    # the mixed kernel on the same work as the plain one (no aperture: every pair)
    p16 = ktm.prepare(raw, sv.dt, fmt="f16", rho=sv.rho_opt, prefold=True)
    img = torch.empty(sv.shape, device=dev, dtype=torch.float32)
    nokw = dict(geo, aperture=0.0)
    for _ in range(3):
        ktm.migrate(traces=p16, image=img, pick="linear", **nokw)
    e0, e1 = _events()
    e0.record()
    for _ in range(a.steps):
        ktm.migrate(traces=p16, image=img, pick="linear", **nokw)
    e1.record()
    torch.cuda.synchronize()
    f16_all = npts * sv.ntr / (e0.elapsed_time(e1) / a.steps * 1e-3) / 1e9
    # plain FP32: the reference-mode kernel (truncating pick, rho-free traces as psktmCPU.c takes them)
    pimg = torch.empty(sv.shape, device=dev, dtype=torch.float32)
    plain_kw = dict(geo, traces=raw, mode="reference", pick="truncate", aperture=0.0, image=pimg)
    for _ in range(3):
        ktm.migrate(**plain_kw)
    e0, e1 = _events()
    e0.record()
    for _ in range(a.steps):
        ktm.migrate(**plain_kw)
    e1.record()
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1) / a.steps
    plain = npts * sv.ntr / (plain_ms * 1e-3) / 1e9
    cpu = None
    if not a.no_cpu_baseline:
        r, cores, kind, sample = cpu_reference_rate(sv, a.cpu_seconds, os.cpu_count() or 1)
        cpu = {"value": r / 1e9, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
        if kind == "reference" and cores > 1:
            r1, _, _, s1 = cpu_reference_rate(sv, a.cpu_seconds / 3, 1)
            cpu["one_thread"] = {"value": r1 / 1e9, "sample": s1}
    print(json.dumps({
        "metric": METRIC, "value": out["f16"]["gpair_s"], "unit": UNIT, "n_gpus": 1,
        "steps": a.steps, "higher_is_better": True, "dtype": "f16 traces, f32 accumulate",
        "data": "synthetic (seeded, device-generated)",
        "config": {"workload": "2-D line: 256 CMPs x 64 offsets (16,384 traces x 1001 samples "
                               "at 4 ms), 256 x 1001 image, aperture 2 km, 2.5-D rho",
                   "weight": "sqrt(j dt) folded into the packed samples"},
        "formats": out, "error_vs": "FP64 device evaluation of the whole image",
        "plain_fp32": {"value": plain, "unit": UNIT, "ms": plain_ms,
                       "mixed_over_plain": {f: out[f]["gpair_s"] / plain for f in out},
                       "f16_no_aperture_gpair_s": f16_all,
                       "mixed_over_plain_same_work": f16_all / plain},
        "cpu_baseline": cpu,
    }), flush=True)


def lsm_main(a):
    """Adjoint and least squares on the 2-D line of 512 CMPs x 64 offsets x 1001
    samples at 4 ms (FP32): the dot-product test <L m, d> = <m, L^T d> with seeded
    Gaussian m and d, 20 CGLS iterations (graph-captured) on data demigrated from a
    seeded sparse reflectivity (5 % non-zeros, N(0,1)), and the Vrms gradient
    against central finite differences of the device image (eps = 1e-3 v)."""
    import torch

    from ktm import synth
    from ktm.inverse import MigrationOperator
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    sv = synth.config4()
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x, dtype=np.float32)).to(dev)  # noqa: E731
    coords = [T(x) for x in (sv.midX, sv.midY, sv.offX, sv.offY)]
    kw = dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt, nt=sv.nt,
              midX=coords[0], midY=coords[1], offX=coords[2], offY=coords[3],
              aperture=sv.aperture)
    # the operator pair's weight: prefolded (default: migration of sqrt(j dt)-folded data,
    # demigration scaled by sqrt(j dt) per sample), the interpolated table, or sqrt.approx
    wt = a.weight
    kw["weight"] = wt
    op = MigrationOperator(velocity=T(sv.velocity1d), **kw)
    rng = np.random.default_rng(4)
    m = T(rng.standard_normal(op.shape))
    d = op.pack(T(rng.standard_normal((sv.ntr, sv.nt))))
    Lm = op.demigrate(m)
    LTd = op.migrate(d)
    lhs = float((Lm.double() * d.double()).sum())
    rhs = float((m.double() * LTd.double()).sum())
    # operator timings
    def timed(fn, n=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n
    demig_ms = timed(lambda: op.demigrate(m, data=Lm))
    mig_ms = timed(lambda: op.migrate(d, image=LTd))
    m_true = T(np.where(rng.uniform(size=op.shape) < 0.05, rng.standard_normal(op.shape), 0.0))
    dobs = op.demigrate(m_true)
    op.least_squares(dobs, 2, use_graph=True)      # warm-up: module loading, first capture
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    model, rn, gn = op.least_squares(dobs, 20, use_graph=True)
    torch.cuda.synchronize()
    lsm_s = time.perf_counter() - t0
    # gradient vs central differences on a band-limited data set
    tr = synth.synthesize_device(sv, device=dev, coords=coords)
    cube = T(np.broadcast_to(sv.velocity1d, op.shape))
    gkw = dict(kw, weight="table")      # the gradient kernel: table weight or prefolded samples
    gop = MigrationOperator(velocity=cube, **gkw)
    packed = gop.pack(tr)
    eps = 1e-3
    opp = MigrationOperator(velocity=cube * (1 + eps), **gkw)
    opm = MigrationOperator(velocity=cube * (1 - eps), **gkw)
    fd = (opp.migrate(packed) - opm.migrate(packed)).double() / (2 * eps * cube.double())
    gpk = gop.packed(packed)
    g = gop.vrms_gradient(gpk).double()
    grad_ms = timed(lambda: gop.vrms_gradient(gpk))
    npairs = op.shape[0] * op.shape[1] * op.shape[2] * sv.ntr
    print(json.dumps({
        "metric": "adjoint / LSM, 2-D line 512 CMPs x 64 offsets x 1001 samples",
        "config": {"workload": "2-D line: 32,768 traces x 1001 samples at 4 ms, 512 x 1001 image, "
                               f"aperture 2 km, FP32, linear pick, {wt} weight"},
        "dot_test": {"lhs": lhs, "rhs": rhs, "rel_diff": abs(lhs - rhs) / abs(lhs)},
        "demigrate_ms": demig_ms, "migrate_ms": mig_ms,
        "demigrate_gpair_s": npairs / (demig_ms * 1e-3) / 1e9,
        "migrate_gpair_s": npairs / (mig_ms * 1e-3) / 1e9,
        "lsm_20": {"seconds": lsm_s, "residual_ratio": float(rn[-1] / rn[0]),
                   "gradient_ratio": float(gn[-1] / gn[0]), "graph": True},
        "vrms_gradient_vs_fd": {"rel_l2": float((g - fd).norm() / fd.norm()), "eps": eps},
        "vrms_gradient_ms": grad_ms,
        "vrms_gradient_gpair_s": npairs / (grad_ms * 1e-3) / 1e9,
    }), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        reference_arm(a)
        return
    if a.config == "batch":
        batch_main(a)
        return
    if a.config == "2d":
        line_main(a)
        return
    if a.config == "lsm":
        lsm_main(a)
        return
    import torch

    import ktm
    from ktm import shard, synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    def allmax(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def allsum(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    # ---- workload: ONE survey; its 200 x 200 image is cut into one output tile per
    # rank (shard.tile_partition) and each rank keeps the traces whose midpoints lie
    # within the aperture of its tile (shard.select_traces, FP64 on the host).  No
    # collective touches the data path; tiles stay on their ranks.
    t_setup = time.perf_counter()
    sv = synth.config2(ntr=a.ntr, seed=2)
    tiles = shard.tile_partition(sv.shape[0], sv.shape[1], world)
    tile = tiles[rank]
    idx = shard.select_traces(sv.midX, sv.midY, tile, sv.imageX, sv.imageY, sv.aperture)
    gx, gy = tile.grids(sv.imageX, sv.imageY)
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x)).to(dev)  # noqa: E731
    coords_all = [T(x) for x in (sv.midX, sv.midY, sv.offX, sv.offY)]
    idx_d = torch.as_tensor(idx.astype(np.int64), device=dev)
    coords = [c.index_select(0, idx_d).contiguous() for c in coords_all]
    vel = shard.tile_velocity(T(sv.velocity), tile)
    vel1 = T(sv.velocity1d)
    raw = torch.empty((len(idx), sv.nt), device=dev, dtype=torch.float32)
    chunk = 100_000
    for k0 in range(0, sv.ntr, chunk):
        k1 = min(sv.ntr, k0 + chunk)
        lo, hi = (int(v) for v in np.searchsorted(idx, [k0, k1]))
        if hi > lo:
            blk = synth.synthesize_device(sv, k0, k1, device=dev, coords=coords_all)
            raw[lo:hi] = blk.index_select(0, idx_d[lo:hi] - k0)
            del blk
    del coords_all
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup

    # a step = one batch of the survey's traces (1/16 by default); this rank takes the
    # batch's traces it selected, which are contiguous in its arrays (idx is sorted)
    nb = a.batches
    bsz = (sv.ntr + nb - 1) // nb
    sbounds = [(b * bsz, min(sv.ntr, (b + 1) * bsz)) for b in range(nb)]
    bounds = [tuple(int(v) for v in np.searchsorted(idx, [b0, b1])) for b0, b1 in sbounds]
    nx, ny, nz = sv.shape
    npts = nx * ny * nz                      # the whole image: pairs count the job's work
    tnx, tny = tile.shape
    tpts = tnx * tny * nz
    stream = torch.cuda.Stream(device=dev)
    image = torch.zeros((tnx, tny, nz), device=dev, dtype=torch.float32)
    pitch = ktm.packed_pitch(sv.nt, a.fmt)
    tdtype = {"f16": torch.float16, "bf16": torch.bfloat16, "f32": torch.float32}[a.fmt]
    maxb = max(1, max(k1 - k0 for k0, k1 in bounds))
    pbuf = torch.empty((maxb, pitch), device=dev, dtype=tdtype)
    pscale = torch.empty(maxb, device=dev, dtype=torch.float32)
    counter = torch.zeros(1, device=dev, dtype=torch.int64)
    geo = dict(imageX=gx, imageY=gy, imageZ=sv.imageZ, dt=sv.dt, pick="linear",
               aperture=sv.aperture)

    # tile shape (tau run x columns per CTA x traces per chunk) from the tuner, timed on
    # this rank's first batch; --tile-run fixes the run and keeps the default shape
    if a.tile_run:
        tile = {"tileRun": a.tile_run, "tileCols": 0, "tileChunk": 0}
    else:
        k0, k1 = bounds[0]
        p0 = ktm.prepare(raw[k0:k1], sv.dt, fmt=a.fmt, rho=sv.rho_opt, prefold=a.weight == "prefold",
                         out=pbuf[:k1 - k0], out_scale=pscale[:k1 - k0])
        tile = ktm.autotune_tile(midX=coords[0][k0:k1], midY=coords[1][k0:k1], offX=coords[2][k0:k1],
                                 offY=coords[3][k0:k1], traces=p0, velocity=vel, image=image,
                                 weight=a.weight, **geo)
        image.zero_()

    def step(i, count=False):
        k0, k1 = bounds[i % nb]
        n = k1 - k0
        with torch.cuda.stream(stream):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            if n == 0:
                e0.record(stream)
                e1.record(stream)
                return e0, e1, n
            p = ktm.prepare(raw[k0:k1], sv.dt, fmt=a.fmt, rho=sv.rho_opt,
                            prefold=a.weight == "prefold",
                            stream=stream, out=pbuf[:n], out_scale=pscale[:n])
            e0.record(stream)
            ktm.migrate(midX=coords[0][k0:k1], midY=coords[1][k0:k1], offX=coords[2][k0:k1],
                        offY=coords[3][k0:k1], traces=p, velocity=vel, image=image,
                        accumulate=(i > 0), stream=stream,
                        pairs_counter=counter if count else None, weight=a.weight,
                        tile=tile, **geo)
            e1.record(stream)
        return e0, e1, n

    # ---- peaks of this GPU (special-function unit and FP32 FMA pipe)
    sq, rs, fm = C.c_double(), C.c_double(), C.c_double()
    ktm._lib.check(ktm.lib().ktmProbePeaks(C.byref(sq), C.byref(rs), C.byref(fm)))

    # ---- warm-up, then K timed steps (events on the launching stream)
    for i in range(a.warmup):
        step(i)
    stream.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    counter.zero_()
    ev0.record(stream)
    kev, traces_done, survey_traces = [], 0, 0
    for i in range(a.steps):
        # the counter costs one atomic add per warp at kernel exit
        e0, e1, n = step(i, count=True)
        kev.append((e0, e1))
        traces_done += n
        b0, b1 = sbounds[i % nb]
        survey_traces += b1 - b0
    ev1.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_rank = ev0.elapsed_time(ev1)
    kernel_ms = sum(e0.elapsed_time(e1) for e0, e1 in kev)
    ms = allmax(ms_rank)
    job_pairs = npts * survey_traces          # the whole image against every trace of the steps
    value = job_pairs / (ms * 1e-3) / 1e9

    # evaluated pairs (after aperture / end-of-trace culling), counted by the kernel
    evaluated = int(counter.item())
    sfu_rate = evaluated * 2 / (kernel_ms * 1e-3)      # two sqrt.approx per evaluated pair
    # in-aperture pairs of the timed batches, counted independently of the kernel
    # (|mid - x| <= aperture over the tile's columns, in FP64; times Nz)
    in_aperture = 0
    cx = (gx.imageStart + gx.imageStep *
          torch.arange(tnx, device=dev, dtype=torch.float64)).repeat_interleave(tny)
    cy = (gy.imageStart + gy.imageStep *
          torch.arange(tny, device=dev, dtype=torch.float64)).repeat(tnx)
    for i in range(a.steps):
        k0, k1 = bounds[i % nb]
        for j0 in range(k0, k1, 4096):
            j1 = min(k1, j0 + 4096)
            dx = coords[0][j0:j1, None].double() - cx[None, :]
            dy = coords[1][j0:j1, None].double() - cy[None, :]
            in_aperture += int(((dx * dx + dy * dy) <= sv.aperture ** 2).sum().item()) * nz
    # per-rank balance: traces kept, pairs evaluated, device time
    stats = torch.tensor([len(idx), evaluated, ms_rank, kernel_ms], device=dev, dtype=torch.float64)
    if dist:
        allstats = [torch.empty_like(stats) for _ in range(world)]
        dist.all_gather(allstats, stats)
    else:
        allstats = [stats]
    per_rank = [{"rank": r, "tile": [tiles[r].ix0, tiles[r].ix1, tiles[r].iy0, tiles[r].iy1],
                 "traces": int(st[0]), "evaluated_pairs": int(st[1]), "ms": float(st[2]),
                 "kernel_ms": float(st[3])}
                for r, st in enumerate(t.cpu().tolist() for t in allstats)]
    evaluated_all = sum(r["evaluated_pairs"] for r in per_rank)
    in_aperture_all = int(allsum(float(in_aperture)))

    # ---- accuracy: one batch through the product path (device rho filter, FP16 packing,
    # fast kernel) into a fresh image, against an FP64 pipeline from the same raw traces:
    # the FP64 rho filter (ktmApplyRhoFilter.m) then the FP64 migration with the weight
    # |tau| sqrt(t) per pair, on a seeded random subgrid of the rank's tile.  Beside it,
    # the kernel alone: the FP64 migration of the FP32 traces the device filter produced.
    err = None
    if not a.skip_error:
        k0, k1 = bounds[0]
        image_keep = image.clone()
        image.zero_()
        step(0)
        stream.synchronize()
        rng = np.random.default_rng(17 + rank)
        xs = np.sort(rng.choice(tnx, size=min(a.err_side, tnx), replace=False))
        ys = np.sort(rng.choice(tny, size=min(a.err_side, tny), replace=False))
        cols = torch.as_tensor((xs[:, None] * tny + ys[None, :]).ravel().astype(np.int32))
        got = image.reshape(tnx * tny, nz)[cols.to(dev).long()].double()
        egeo = dict(columns=cols, midX=coords[0][k0:k1], midY=coords[1][k0:k1],
                    offX=coords[2][k0:k1], offY=coords[3][k0:k1], velocity=vel, **geo)
        f64 = rho_filter_f64(raw[k0:k1], sv.dt, sv.rho_opt)
        ref = ktm.migrate_columns_f64(traces=f64, **egeo).double()
        del f64
        p32 = ktm.prepare(raw[k0:k1], sv.dt, fmt="f32", rho=sv.rho_opt, prefold=False)
        ref_k = ktm.migrate_columns_f64(traces=p32, **egeo).double()
        del p32
        err = {"rel_l2": allmax(float((got - ref).norm() / ref.norm())),
               "max_rel": allmax(float((got - ref).abs().max() / ref.abs().max())),
               "vs": "FP64 pipeline from the raw traces: FP64 rho filter (ktmApplyRhoFilter.m, "
                     "3-D i*omega), then FP64 migration (linear pick, |tau| sqrt(t) per pair)",
               "sample": (f"seeded random {len(xs)}x{len(ys)}x{nz} subgrid of each rank's tile, "
                          f"batch 0 ({sbounds[0][1] - sbounds[0][0]} survey traces); max over ranks"),
               "kernel_only": {"rel_l2": allmax(float((got - ref_k).norm() / ref_k.norm())),
                               "max_rel": allmax(float((got - ref_k).abs().max() / ref_k.abs().max())),
                               "vs": "FP64 migration of the device-filtered FP32 traces"}}
        image.copy_(image_keep)

    # ---- plain FP32 path (psktmCPU.c arithmetic, bit-exact kernel) on part of a batch
    k0p, k1p = bounds[0]
    kp = max(1, min(k1p - k0p, bsz // 4)) if not a.skip_plain else 64
    kp = min(kp, raw.shape[0])
    plain_kw = dict(imageX=gx, imageY=gy, imageZ=sv.imageZ, dt=sv.dt,
                    midX=coords[0][:kp], midY=coords[1][:kp], offX=coords[2][:kp],
                    offY=coords[3][:kp], traces=raw[:kp], velocity=vel1, mode="reference",
                    pick="truncate", stream=stream)
    ks = min(64, kp)
    small = dict(plain_kw, midX=coords[0][:ks], midY=coords[1][:ks], offX=coords[2][:ks],
                 offY=coords[3][:ks], traces=raw[:ks])
    pimg = torch.empty((tnx, tny, nz), device=dev, dtype=torch.float32)
    ktm.migrate(image=pimg, **small)
    stream.synchronize()
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pe0.record(stream)
    ktm.migrate(image=pimg, **plain_kw)
    pe1.record(stream)
    stream.synchronize()
    plain_ms = pe0.elapsed_time(pe1)
    plain_rate = tpts * kp / (plain_ms * 1e-3) / 1e9
    del pimg

    # ---- end to end through the C ABI with host buffers (pinned), per step: this rank's
    # traces of batch 0, their coordinates and the tile's Vrms host->device, the tile
    # image device->host; as many steps as the device-timed measurement
    e2e = None
    e2e_steps = a.steps if a.e2e_steps is None else a.e2e_steps
    if e2e_steps > 0:
        k0, k1 = bounds[0]
        n = k1 - k0
        h_tr = torch.empty((n, sv.nt), dtype=torch.float32, pin_memory=True)
        h_tr.copy_(raw[k0:k1])
        h_c = [torch.empty(n, dtype=torch.float32, pin_memory=True).copy_(c[k0:k1]) for c in coords]
        h_v = torch.empty(vel.shape, dtype=torch.float32, pin_memory=True).copy_(vel)
        h_img = torch.empty((tnx, tny, nz), dtype=torch.float32, pin_memory=True)
        hk = dict(midX=h_c[0].numpy(), midY=h_c[1].numpy(), offX=h_c[2].numpy(),
                  offY=h_c[3].numpy(), traces=h_tr.numpy(), velocity=h_v.numpy(),
                  image=h_img.numpy(), rho=sv.rho_opt, pack_format=a.fmt, weight=a.weight,
                  stream=stream, **geo)
        ktm.migrate(**hk)   # warm-up
        if dist:
            dist.barrier()
        he0, he1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        he0.record(stream)
        for _ in range(e2e_steps):
            ktm.migrate(**hk)
        he1.record(stream)
        stream.synchronize()
        wall = time.perf_counter() - t0
        e_ms = allmax(max(he0.elapsed_time(he1), wall * 1e3) / e2e_steps)
        h2d = n * sv.nt * 4 + 4 * n * 4 + vel.numel() * 4
        e2e = {"value": npts * (sbounds[0][1] - sbounds[0][0]) / (e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": int(allsum(float(h2d))),
               "d2h_bytes_per_step": int(allsum(float(tpts * 4))),
               "steps": e2e_steps,
               "per_step": "each rank's traces of one batch through ktmMigrate, host memory; "
                           "max over ranks"}

    # ---- CPU baseline (rank 0, N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        sub = synth.config2(ntr=8192, seed=2)
        r, cores, kind, sample = cpu_reference_rate(sub, a.cpu_seconds, os.cpu_count() or 1)
        cpu = {"value": r / 1e9, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
        if kind == "reference" and cores > 1:
            # the one-thread run of the same code (the configuration reference mode matches
            # bit for bit; the OpenMP loop races on image[] with more threads)
            r1, _, _, s1 = cpu_reference_rate(sub, a.cpu_seconds / 3, 1)
            cpu["one_thread"] = {"value": r1 / 1e9, "sample": s1}

    if rank == 0:
        per_launch_ms = kernel_ms / a.steps
        # binding roofline: the special-function unit.  Fixed algorithmic work per
        # pair: 3 MUFU ops (2 DSR square roots + 1 for the weight sqrt(t)) and 17 FP32
        # flops, so the pair ceiling is min(MUFU peak / 3, FP32 peak / 17); both
        # peaks measured now on this GPU (ktmProbePeaks).  Rank 0's own kernel.
        eval_rate = evaluated / (kernel_ms * 1e-3)
        if cpu:
            # psktmCPU.c evaluates every pair; the GPU kernel skips pairs outside the
            # aperture and past the trace end, so beside the raw ratio: evaluated pairs
            cpu["gpu_over_cpu"] = {"raw": value / cpu["value"],
                                   "same_work": eval_rate / 1e9 / cpu["value"],
                                   "note": "raw: value / this baseline; same_work: the GPU "
                                           "kernel's evaluated (in-aperture) pairs/s / this "
                                           "baseline, which evaluates every pair"}
        # our kernels per step: ktmPrepareTraces (1) + the migration, one launch per
        # trace block of at most 40 MB of packed samples (ktm_fast.cu)
        esz = 4 if a.fmt == "f32" else 2
        blk = max(1024, (40 << 20) // (pitch * esz))
        launches = sum(1 + -(-(bounds[i % nb][1] - bounds[i % nb][0]) // blk)
                       for i in range(a.steps) if bounds[i % nb][1] > bounds[i % nb][0])
        pair_peak = min(sq.value / 3.0, 2.0 * fm.value / 17.0)
        rank_b = bounds[0][1] - bounds[0][0]
        balance = [r["evaluated_pairs"] for r in per_rank]
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None, "dtype": f"{a.fmt} traces, f32 accumulate",
            "data": "synthetic (seeded, device-generated)",
            "config": {"workload": WORKLOAD, "traces": sv.ntr, "image": [nx, ny, nz],
                       "batch_traces": bsz, "trace_format": a.fmt, "rho": "3D (i*omega)",
                       "pick": "linear", "aperture_m": sv.aperture, "tile": tile,
                       "weight": {"prefold": "sqrt(j dt) folded into the packed samples",
                                  "table": "sqrt(t) from the interpolated sqrt(j dt) table",
                                  "sqrt": "sqrt(t) by sqrt.approx per pair"}[a.weight],
                       "l2": "each step reads a new batch of traces (375 MB raw at N=1, > 126 MB L2)",
                       "parallelism": (f"output tiles: the {nx}x{ny} image of one survey cut into "
                                       f"{world} tile(s) (ktm.shard.tile_partition), each rank "
                                       "migrating the traces its tile's aperture selects "
                                       "(FP64 host cull); no collective in the data path")},
            "per_rank": per_rank,
            "imbalance": (max(balance) / (sum(balance) / len(balance))) if sum(balance) else None,
            "plain_fp32": {"value": plain_rate, "unit": UNIT,
                           "kernel": "bit-exact psktmCPU.c arithmetic (no aperture: every pair)",
                           "sample": f"{kp} traces x rank 0's tile, 1-D velocity",
                           "mixed_over_plain": tpts * traces_done / (ms_rank * 1e-3) / 1e9
                                               / plain_rate,
                           "mixed_over_plain_same_work": eval_rate / 1e9 / plain_rate,
                           "same_work_note": "evaluated (in-aperture) pairs/s of the mixed "
                                             "kernel over the plain kernel's pairs/s"},
            "error": err,
            "pairs": {"raw_per_step": npts * bsz, "evaluated_fraction": evaluated_all / max(1, job_pairs),
                      "evaluated_rate_gpair_s": eval_rate / 1e9,
                      "in_aperture_fraction": in_aperture_all / max(1, job_pairs),
                      "note": "evaluated = in aperture and not past the trace end (kernel "
                              "counter, all ranks); in_aperture counted separately in FP64"},
            "roofline": {"bound": "sfu", "achieved": eval_rate / 1e9, "peak": pair_peak / 1e9,
                         "unit": "Gpair/s", "frac": eval_rate / pair_peak,
                         "traffic": MIGRATE_DRAM_BYTES_PER_TRACE * rank_b,
                         "algorithmic_bytes": rank_b * pitch * esz + tpts * 4,
                         "definition": "evaluated pairs/s over the migrate kernel's event time; "
                                       "peak = min(MUFU/3, FP32 flops/17) pairs/s with the "
                                       "MUFU (sqrt.approx) and FFMA throughputs measured now",
                         "sfu_issued": {"achieved_tsqrt_s": sfu_rate / 1e12,
                                        "peak_tsqrt_s": sq.value / 1e12,
                                        "frac": sfu_rate / sq.value,
                                        "note": ("2 sqrt.approx per pair, sqrt(t) prefolded into "
                                                 "the samples" if a.weight == "prefold" else
                                                 "2 sqrt.approx per pair, plus the weight's "
                                                 "table lookup or third sqrt.approx")},
                         "traffic_note": MIGRATE_DRAM_NOTE,
                         "kernel_ms_per_step": per_launch_ms},
            "peaks_measured": {"sqrt_t_s": sq.value / 1e12, "rsqrt_t_s": rs.value / 1e12,
                               "ffma_t_s": fm.value / 1e12},
            "clocks": clk,
            "e2e": e2e,
            "gpu_launches": launches,
            "cpu_baseline": cpu,
            "setup_s": setup_s,
        }
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
