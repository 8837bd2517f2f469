"""The reference arm of bench.py runs on the host alone: the reference's own
psktmCPU.c (oracle/_ref, or the oracle restatement where it was not built) on a
bounded sample of the 3-D workload.  Checks the JSON line it prints carries the
keys the benchmark contract asks for, with a short per-step budget."""
from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    env = dict(os.environ, RANK="0", CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "2", "--warmup", "1", "--ref-step-seconds", "0.5"],
                         capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "Gpair/s" and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 1 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["kind"] in ("reference", "port")
    assert d["e2e"] == {"value": d["value"], "unit": "Gpair/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0", "--ref-step-seconds", "0.5"],
                         capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert out.returncode == 0 and not out.stdout.strip()


def _bench():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import bench
    return bench


def test_cpu_sample_fills_every_thread():
    """The CPU sample is whole waves of the OpenMP team (psktmCPU.c:56 spreads its
    trace loop over the threads) with at least eight traces per thread."""
    from ktm import synth
    bench = _bench()
    sv = synth.areal_survey(ntr=600, side=1500.0, maxoff=800.0, nx=12, ny=10, dxy=25.0,
                            nt=300, dt=0.004, nz=300, nscat=3, freq=25.0, noise=0.05,
                            aperture=1000.0, vtop=1500.0, vbot=2500.0, lateral=0.0, rho_opt=3,
                            seed=3, name="sizing")
    for threads in (1, 3, 4):
        ref = bench.CpuReference(sv, 0.05, threads)
        assert ref.ntr % ref.threads == 0 and ref.ntr >= 8 * ref.threads
        assert ref.rate() > 0


def test_bench_rho_f64_matches_oracle_restatement():
    """The bench's FP64 rho filter (torch) against oracle/rho.py (numpy), all three
    filters, an odd and a power-of-two trace length."""
    import numpy as np
    import torch

    import rho
    bench = _bench()
    rng = np.random.default_rng(9)
    for m in (1501, 1024, 7):
        x = rng.standard_normal((5, m))
        for opt in (1, 2, 3):
            got = bench.rho_filter_f64(torch.as_tensor(x), 0.002, opt).numpy()
            want = rho.rho_filter_traces(x, 0.002 * 1e6, opt)
            assert np.allclose(got, want, rtol=1e-12, atol=1e-9 * np.abs(want).max()), (m, opt)
