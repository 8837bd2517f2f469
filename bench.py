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
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-plain", action="store_true", help="skip the plain FP32 comparison")
    ap.add_argument("--skip-error", action="store_true", help="skip the FP64 error check")
    ap.add_argument("--config", default="3d", choices=["3d", "batch", "2d", "lsm"],
                    help="3d: the headline workload; batch: 64 target-oriented jobs in one "
                         "persistent launch")
    ap.add_argument("--jobs", type=int, default=64)
    ap.add_argument("--lsm-jobs", type=int, default=4)
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
def cpu_reference_rate(sv, seconds: float, threads: int):
    """The reference's psktmCPU.c (oracle/_ref, compiled unmodified) or, where it
    was never built, the oracle's single-thread restatement, on a bounded sample
    of the workload: the full image against the first T traces, T sized so the
    run takes about ``seconds``.  Returns (pairs/s, cores, kind, sample)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    kind = "reference" if oracle.ref_available() else "port"
    if kind == "port":
        threads = 1
    nx, ny, nz = sv.shape

    def run(ntr):
        tr = np.random.default_rng(5).standard_normal((ntr, sv.nt)).astype(np.float32)
        args = (sv.imageX, sv.imageY, sv.imageZ, sv.dt, sv.midX[:ntr], sv.midY[:ntr],
                sv.offX[:ntr], sv.offY[:ntr], tr, sv.velocity1d)
        t0 = time.perf_counter()
        if kind == "reference":
            oracle.migrate_reference_c(*args, threads=threads)
        else:
            oracle.migrate_ref32(*args)
        return time.perf_counter() - t0

    g = oracle.grid
    sv.imageX, sv.imageY, sv.imageZ = (g(a.imagePnts, a.imageStep, a.imageStart)
                                       for a in (sv.imageX, sv.imageY, sv.imageZ))
    t1 = run(1)
    ntr = int(max(1, min(sv.ntr, seconds / max(t1, 1e-3))))
    dt = run(ntr)
    pairs = nx * ny * nz * ntr
    sample = (f"full {nx}x{ny}x{nz} image x first {ntr} traces ({pairs:.3e} pairs), "
              f"1-D RMS velocity, {threads} OpenMP threads" if kind == "reference" else
              f"full image x first {ntr} traces, single-thread oracle restatement")
    return pairs / dt, threads, kind, sample


def reference_arm(a):
    """--impl reference: the reference's CPU implementation of the path, rank 0."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from ktm import synth
    sv = synth.config2(ntr=20000)
    threads = os.cpu_count() or 1
    rates = []
    budget = (a.ref_step_seconds if a.ref_step_seconds is not None
              else max(2.0, 150.0 / max(1, a.steps + a.warmup)))
    info = None
    for i in range(a.warmup + a.steps):
        r, cores, kind, sample = cpu_reference_rate(sv, budget, threads)
        if i >= a.warmup:
            rates.append(r)
        info = (cores, kind, sample)
    v = float(np.mean(rates)) / 1e9
    cores, kind, sample = info
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "per_step": "bounded CPU sample, see cpu_baseline"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------------------------------
def batch_main(a):
    """64 target-oriented jobs in ONE persistent launch (ktmMigrateBatch).

    Patch sides log-uniform in [16, 128] bins of 12.5 m, 751 tau samples (t0 at
    4 ms); trace counts log-uniform in [1e4, 5e5]; per job, sources and receivers
    uniform over the patch grown by the 2 km aperture, offsets <= 3150 m, the
    line survey's Vrms(t0) = 1500 + 0.5 t0[ms], 25 Hz Ricker diffractions from
    20 scatterers plus sigma 0.05 noise, 2.5-D rho filter, BF16 traces with an
    FP32 scale and sqrt(j dt) folded in, FP32 accumulation, tau-run length from
    ktmAutotune.  Then the
    error of sampled jobs against the FP64 device evaluation, and 10-iteration
    CGLS (one iteration captured in a CUDA graph) on the smallest jobs."""
    import torch

    import ktm
    from ktm import synth
    from ktm.inverse import MigrationOperator
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(55)
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x, dtype=np.float32)).to(dev)  # noqa: E731
    jobs, surveys = [], []
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
        packed = ktm.prepare(raw, sv.dt, fmt="bf16", rho=sv.rho_opt, prefold=True)
        del raw
        jobs.append(dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt,
                         midX=coords[0], midY=coords[1], offX=coords[2], offY=coords[3],
                         traces=packed, velocity=T(sv.velocity1d), pick="linear",
                         aperture=sv.aperture,
                         image=torch.empty(sv.shape, device=dev, dtype=torch.float32)))
        surveys.append(sv)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    run = ktm.autotune(**jobs[0])
    for kw in jobs:
        kw["tile_run"] = run
    pairs = sum(s.pairs for s in surveys)
    ktm.migrate_batch(jobs)                                   # warm-up
    torch.cuda.synchronize()
    times = []
    for _ in range(max(1, a.steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ktm.migrate_batch(jobs)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = float(np.median(times))
    # per-job error on sampled jobs and columns
    errs = []
    for j in rng.choice(len(jobs), size=min(8, len(jobs)), replace=False):
        sv, kw = surveys[j], jobs[j]
        raw = synth.synthesize_device(sv, device=dev, coords=[kw[k] for k in ("midX", "midY", "offX", "offY")])
        p32 = ktm.prepare(raw, sv.dt, fmt="f32", rho=sv.rho_opt, prefold=False)
        del raw
        nx, ny, nz = sv.shape
        cols = torch.as_tensor(rng.choice(nx * ny, size=min(32, nx * ny), replace=False).astype(np.int32))
        ref = ktm.migrate_columns_f64(columns=cols, **{**kw, "traces": p32, "image": None,
                                                       "tile_run": 0}).double()
        got = kw["image"].reshape(nx * ny, nz)[cols.to(dev).long()].double()
        errs.append(float((got - ref).norm() / ref.norm()))
    # 10-iteration CGLS per job (graph-captured iteration) on the smallest jobs
    lsm = []
    for j in np.argsort([s.pairs for s in surveys])[: a.lsm_jobs]:
        sv, kw = surveys[j], jobs[j]
        op = MigrationOperator(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt,
                               nt=sv.nt, midX=kw["midX"], midY=kw["midY"], offX=kw["offX"],
                               offY=kw["offY"], velocity=kw["velocity"], aperture=sv.aperture)
        d = op.pack(kw["traces"].unpacked())
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        _, rn, _ = op.least_squares(d, 10, use_graph=True)
        lsm.append({"job": int(j), "traces": sv.ntr, "image": list(sv.shape),
                    "residual_ratio": float(rn[-1] / rn[0]), "seconds": time.perf_counter() - t1})
    print(json.dumps({
        "metric": METRIC, "config": {"workload": f"batched: {len(jobs)} jobs in one persistent launch",
                                     "patch_sides": [s.shape[0] for s in surveys],
                                     "traces": [s.ntr for s in surveys], "nz": 751,
                                     "trace_format": "bf16", "tile_run": run,
                                     "weight": "sqrt(j dt) folded into the packed samples"},
        "value": pairs / (ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_launch": ms, "pairs": pairs,
        "steps": len(times), "error_rel_l2": {"max": max(errs), "median": float(np.median(errs)),
                                               "jobs": len(errs), "vs": "FP64 device, 32 columns per job"},
        "lsm_10_iterations": lsm, "setup_s": setup_s,
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
    g = gop.vrms_gradient(gop.packed(packed)).double()
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
    from ktm import synth

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

    # ---- workload: each rank images its own 5 x 5 km tile (weak scaling, no data-path
    # collective); rank r's survey is the same recipe with seed 2 + r
    t_setup = time.perf_counter()
    sv = synth.config2(ntr=a.ntr, seed=2 + rank)
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x)).to(dev)  # noqa: E731
    coords = [T(x) for x in (sv.midX, sv.midY, sv.offX, sv.offY)]
    vel = T(sv.velocity)
    vel1 = T(sv.velocity1d)
    raw = torch.empty((sv.ntr, sv.nt), device=dev, dtype=torch.float32)
    chunk = 100_000
    for k0 in range(0, sv.ntr, chunk):
        synth.synthesize_device(sv, k0, min(sv.ntr, k0 + chunk), device=dev, coords=coords,
                                out=raw[k0:min(sv.ntr, k0 + chunk)])
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup

    nb = a.batches
    bsz = (sv.ntr + nb - 1) // nb
    bounds = [(b * bsz, min(sv.ntr, (b + 1) * bsz)) for b in range(nb)]
    nx, ny, nz = sv.shape
    npts = nx * ny * nz
    stream = torch.cuda.Stream(device=dev)
    image = torch.zeros(sv.shape, device=dev, dtype=torch.float32)
    pitch = ktm.packed_pitch(sv.nt, a.fmt)
    tdtype = {"f16": torch.float16, "bf16": torch.bfloat16, "f32": torch.float32}[a.fmt]
    pbuf = torch.empty((bsz, pitch), device=dev, dtype=tdtype)
    pscale = torch.empty(bsz, device=dev, dtype=torch.float32)
    counter = torch.zeros(1, device=dev, dtype=torch.int64)

    def step(i, count=False):
        k0, k1 = bounds[i % nb]
        n = k1 - k0
        with torch.cuda.stream(stream):
            p = ktm.prepare(raw[k0:k1], sv.dt, fmt=a.fmt, rho=sv.rho_opt,
                            prefold=a.weight == "prefold",
                            stream=stream, out=pbuf[:n], out_scale=pscale[:n])
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ktm.migrate(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt,
                        midX=coords[0][k0:k1], midY=coords[1][k0:k1], offX=coords[2][k0:k1],
                        offY=coords[3][k0:k1], traces=p, velocity=vel, image=image,
                        pick="linear", aperture=sv.aperture, accumulate=(i > 0), stream=stream,
                        pairs_counter=counter if count else None, weight=a.weight,
                        tile_run=a.tile_run)
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
    kev, traces_done = [], 0
    for i in range(a.steps):
        # the counter costs one atomic add per warp at kernel exit
        e0, e1, n = step(i, count=True)
        kev.append((e0, e1))
        traces_done += n
    ev1.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    kernel_ms = sum(e0.elapsed_time(e1) for e0, e1 in kev)
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    pairs_rank = npts * traces_done
    value = pairs_rank * world / (ms * 1e-3) / 1e9

    # evaluated pairs (after aperture / end-of-trace culling), counted by the kernel
    evaluated = int(counter.item())
    sfu_rate = evaluated * 2 / (kernel_ms * 1e-3)      # two sqrt.approx per evaluated pair
    # in-aperture pairs of the timed batches, counted independently of the kernel
    # (|mid - x| <= aperture over all image columns, in FP64; times Nz)
    in_aperture = 0
    cx = (sv.imageX.imageStart + sv.imageX.imageStep *
          torch.arange(nx, device=dev, dtype=torch.float64)).repeat_interleave(ny)
    cy = (sv.imageY.imageStart + sv.imageY.imageStep *
          torch.arange(ny, device=dev, dtype=torch.float64)).repeat(nx)
    for i in range(a.steps):
        k0, k1 = bounds[i % nb]
        for j0 in range(k0, k1, 4096):
            j1 = min(k1, j0 + 4096)
            dx = coords[0][j0:j1, None].double() - cx[None, :]
            dy = coords[1][j0:j1, None].double() - cy[None, :]
            in_aperture += int(((dx * dx + dy * dy) <= sv.aperture ** 2).sum().item()) * nz

    # ---- accuracy: one batch, fresh image, vs FP64 device evaluation (rho-filtered
    # FP32 input, weight |tau| sqrt(t) per pair) on sampled columns
    rel_l2 = max_err = None
    ncols_err = (0, 0)
    if not a.skip_error:
        k0, k1 = bounds[0]
        image_keep = image.clone()
        image.zero_()
        step(0)
        stream.synchronize()
        p32 = ktm.prepare(raw[k0:k1], sv.dt, fmt="f32", rho=sv.rho_opt, prefold=False)
        rng = np.random.default_rng(17)
        xs = np.sort(rng.choice(nx, size=min(a.err_side, nx), replace=False))
        ys = np.sort(rng.choice(ny, size=min(a.err_side, ny), replace=False))
        cols = torch.as_tensor((xs[:, None] * ny + ys[None, :]).ravel().astype(np.int32))
        ncols_err = (len(xs), len(ys))
        ref = ktm.migrate_columns_f64(
            columns=cols, imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt,
            midX=coords[0][k0:k1], midY=coords[1][k0:k1], offX=coords[2][k0:k1],
            offY=coords[3][k0:k1], traces=p32, velocity=vel, pick="linear", aperture=sv.aperture)
        # p32 is not prefolded: the FP64 evaluation applies |tau| sqrt(t) per pair
        got = image.reshape(nx * ny, nz)[cols.to(dev).long()].double()
        ref = ref.double()
        rel_l2 = float((got - ref).norm() / ref.norm())
        max_err = float((got - ref).abs().max() / ref.abs().max())
        del p32
        image.copy_(image_keep)

    # ---- plain FP32 path (psktmCPU.c arithmetic, bit-exact kernel) on part of a batch
    kp = max(1, bsz // 4) if not a.skip_plain else 64
    plain_kw = dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt,
                    midX=coords[0][:kp], midY=coords[1][:kp], offX=coords[2][:kp],
                    offY=coords[3][:kp], traces=raw[:kp], velocity=vel1, mode="reference",
                    pick="truncate", stream=stream)
    small = dict(plain_kw, midX=coords[0][:64], midY=coords[1][:64], offX=coords[2][:64],
                 offY=coords[3][:64], traces=raw[:64])
    pimg = torch.empty(sv.shape, device=dev, dtype=torch.float32)
    ktm.migrate(image=pimg, **small)
    stream.synchronize()
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pe0.record(stream)
    ktm.migrate(image=pimg, **plain_kw)
    pe1.record(stream)
    stream.synchronize()
    plain_ms = pe0.elapsed_time(pe1)
    plain_rate = npts * kp / (plain_ms * 1e-3) / 1e9
    del pimg

    # ---- end to end through the C ABI with host buffers (pinned), per batch:
    # traces, coordinates, velocity cube host->device, image device->host
    e2e = None
    if a.e2e_steps > 0:
        k0, k1 = bounds[0]
        n = k1 - k0
        h_tr = torch.empty((n, sv.nt), dtype=torch.float32, pin_memory=True)
        h_tr.copy_(raw[k0:k1])
        h_c = [torch.empty(n, dtype=torch.float32, pin_memory=True).copy_(c[k0:k1]) for c in coords]
        h_v = torch.empty(vel.shape, dtype=torch.float32, pin_memory=True).copy_(vel)
        h_img = torch.empty(sv.shape, dtype=torch.float32, pin_memory=True)
        hk = dict(imageX=sv.imageX, imageY=sv.imageY, imageZ=sv.imageZ, dt=sv.dt,
                  midX=h_c[0].numpy(), midY=h_c[1].numpy(), offX=h_c[2].numpy(),
                  offY=h_c[3].numpy(), traces=h_tr.numpy(), velocity=h_v.numpy(),
                  image=h_img.numpy(), pick="linear", aperture=sv.aperture, rho=sv.rho_opt,
                  pack_format=a.fmt, weight=a.weight, stream=stream)
        ktm.migrate(**hk)   # warm-up
        he0, he1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        he0.record(stream)
        for _ in range(a.e2e_steps):
            ktm.migrate(**hk)
        he1.record(stream)
        stream.synchronize()
        wall = time.perf_counter() - t0
        e_ms = max(he0.elapsed_time(he1), wall * 1e3) / a.e2e_steps
        if dist:                                   # the slowest rank's time, as for value
            t = torch.tensor([e_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e_ms = float(t.item())
        h2d = n * sv.nt * 4 + 4 * n * 4 + vel.numel() * 4
        e2e = {"value": npts * n / (e_ms * 1e-3) / 1e9 * world, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(npts * 4),
               "steps": a.e2e_steps, "per_step": "one batch through ktmMigrate, host memory"}

    # ---- CPU baseline (rank 0, N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        sub = synth.config2(ntr=4096, seed=2)
        r, cores, kind, sample = cpu_reference_rate(sub, a.cpu_seconds, os.cpu_count() or 1)
        cpu = {"value": r / 1e9, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}
        if kind == "reference" and cores > 1:
            # the one-thread run of the same code (the configuration reference mode matches
            # bit for bit; the OpenMP loop races on image[] with more threads)
            r1, _, _, s1 = cpu_reference_rate(sub, a.cpu_seconds / 3, 1)
            cpu["one_thread"] = {"value": r1 / 1e9, "sample": s1}

    # DRAM bytes of one step from the ncu capture summarised in profiles/ (one step of
    # the same workload), scaled to this batch by its traces
    traffic = None
    tf = os.path.join(ROOT, "profiles", "migrate_fast_traffic.txt")
    if os.path.exists(tf):
        kv = dict(line.split(":", 1) for line in open(tf) if ":" in line and not line.startswith("#"))
        try:
            traffic = float(kv["dram_bytes_per_step"]) / float(kv["traces_per_step"]) * bsz
        except (KeyError, ValueError):
            traffic = None

    if rank == 0:
        per_launch_ms = kernel_ms / a.steps
        # binding roofline: the special-function unit.  Fixed algorithmic work per
        # pair: 3 MUFU ops (2 DSR square roots + 1 for the weight sqrt(t)) and 17 FP32
        # flops, so the pair ceiling is min(MUFU peak / 3, FP32 peak / 17); both
        # peaks measured now on this GPU (ktmProbePeaks)
        eval_rate = evaluated / (kernel_ms * 1e-3)
        # our kernels per step: ktmPrepareTraces (1) + the migration, one launch per
        # trace block of at most 40 MB of packed samples (ktm_fast.cu)
        esz = 4 if a.fmt == "f32" else 2
        blk = max(1024, (40 << 20) // (pitch * esz))
        nblk = -(-bsz // blk)
        launches = a.steps * (1 + nblk)
        pair_peak = min(sq.value / 3.0, 2.0 * fm.value / 17.0)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": f"{a.fmt} traces, f32 accumulate",
            "data": "synthetic (seeded, device-generated)",
            "config": {"workload": WORKLOAD, "traces": sv.ntr, "image": [nx, ny, nz],
                       "batch_traces": bsz, "trace_format": a.fmt, "rho": "3D (i*omega)",
                       "pick": "linear", "aperture_m": sv.aperture,
                       "weight": {"prefold": "sqrt(j dt) folded into the packed samples",
                                  "table": "sqrt(t) from the interpolated sqrt(j dt) table",
                                  "sqrt": "sqrt(t) by sqrt.approx per pair"}[a.weight],
                       "l2": "each step reads a new 375 MB batch (> 126 MB L2)",
                       "parallelism": f"{world} GPU(s), one image tile per GPU, no collective"},
            "plain_fp32": {"value": plain_rate, "unit": UNIT,
                           "kernel": "bit-exact psktmCPU.c arithmetic (no aperture: every pair)",
                           "sample": f"{kp} traces x full image, 1-D velocity",
                           "mixed_over_plain": value / world / plain_rate,
                           "mixed_over_plain_same_work": (evaluated / (kernel_ms * 1e-3) / 1e9)
                                                         / plain_rate,
                           "same_work_note": "evaluated (in-aperture) pairs/s of the mixed "
                                             "kernel over the plain kernel's pairs/s"},
            "error": {"rel_l2": rel_l2, "max_rel": max_err, "vs": "FP64 device evaluation",
                      "sample": f"seeded random {ncols_err[0]}x{ncols_err[1]}x{nz} subgrid, "
                                f"batch 0 ({bsz} traces)"},
            "pairs": {"raw_per_step": npts * bsz, "evaluated_fraction": evaluated / max(1, pairs_rank),
                      "evaluated_rate_gpair_s": evaluated / (kernel_ms * 1e-3) / 1e9,
                      "in_aperture_fraction": in_aperture / max(1, pairs_rank),
                      "note": "evaluated = in aperture and not past the trace end (kernel "
                              "counter); in_aperture counted separately in FP64"},
            "roofline": {"bound": "sfu", "achieved": eval_rate / 1e9, "peak": pair_peak / 1e9,
                         "unit": "Gpair/s", "frac": eval_rate / pair_peak,
                         "traffic": traffic,
                         "algorithmic_bytes": bsz * pitch * (4 if a.fmt == "f32" else 2) + npts * 4,
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
                         "traffic_note": "DRAM read+write of one step (5 launches of the "
                                         "kernel, one per 40 MB trace block) from one ncu "
                                         "capture, scaled by traces",
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
