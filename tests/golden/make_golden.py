"""Generate the golden fixtures of the PSTM hot path from the reference's own code.

    make -C oracle            # builds oracle/_ref/libktm_ref.so from the reference sources
    python tests/golden/make_golden.py

Each fixture holds seeded inputs and the output of the reference's
ktmMigrationCPU (src/psktmCPU.c, compiled unmodified, run with ONE OpenMP
thread because the reference loop races on image[] with more,
psktmCPU.c:56-85) or of its ktmIBM32toIEEE (src/ioFunctions.c:4-40).  The
fixtures pin the oracle restatement and the CUDA kernels on machines where the
reference sources are absent.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "seismic-migration_b200"))

import oracle  # noqa: E402
from ktm import synth  # noqa: E402


def _grid(a):
    return oracle.grid(*a)


def run_case(path, gx, gy, gz, dt, midx, midy, offx, offy, traces, vel):
    g = [tuple(v) for v in (gx, gy, gz)]
    img = oracle.migrate_reference_c(_grid(gx), _grid(gy), _grid(gz), dt, midx, midy, offx,
                                     offy, traces, vel, threads=1)
    np.savez_compressed(path, gx=np.array(g[0]), gy=np.array(g[1]), gz=np.array(g[2]),
                        dt=np.float32(dt), midX=midx, midY=midy, offX=offx, offY=offy,
                        traces=traces, velocity=vel, image=img)
    print(os.path.basename(path), img.shape, float(np.abs(img).max()))


def main():
    rng = np.random.default_rng(20240601)
    # 1. small 2-D line with diffraction data (the structure of the benchmark line)
    sv = synth.line_survey(ncmp=24, noff=8, doff=150.0, nt=200, dt=0.004, nz=150, nscat=4,
                           seed=11)
    tr = synth.synthesize(sv)
    run_case(os.path.join(HERE, "ref_line_small.npz"), (24, 12.5, 0.0), (1, 1.0, 0.0),
             (150, 0.002, 0.0), sv.dt, sv.midX, sv.midY, sv.offX, sv.offY, tr, sv.velocity1d)

    # 2. small areal survey, random data, 2-D image grid, non-zero axis origins
    ntr, nt = 160, 128
    mid = rng.uniform(-300.0, 300.0, (ntr, 2)).astype(np.float32)
    off = rng.uniform(-400.0, 400.0, (ntr, 2)).astype(np.float32)
    tr = rng.standard_normal((ntr, nt)).astype(np.float32)
    vel = np.linspace(1600.0, 3000.0, 90).astype(np.float32)
    run_case(os.path.join(HERE, "ref_areal_small.npz"), (7, 40.0, -120.0), (5, 55.0, -100.0),
             (90, 0.003, 0.01), 0.004, mid[:, 0], mid[:, 1], off[:, 0], off[:, 1], tr, vel)

    # 3. zero-offset traces on the image points: t = 2 tau lands on sample
    #    boundaries (it = (int)(t/dt) exactly at integers), sample 0 exclusion,
    #    tau = 0 row (0/0 weights never used), last-sample exclusion
    nx, nt = 9, 64
    xs = np.arange(nx, dtype=np.float32) * 10.0
    midx = np.concatenate([xs, xs + 5.0]).astype(np.float32)
    z = np.zeros_like(midx)
    tr = (np.arange(2 * nx * nt, dtype=np.float32).reshape(2 * nx, nt) % 17 - 8.0).astype(np.float32)
    vel = np.full(70, 2000.0, np.float32)
    run_case(os.path.join(HERE, "ref_zero_offset.npz"), (nx, 10.0, 0.0), (1, 1.0, 0.0),
             (70, 0.002, 0.0), 0.004, midx, z, z, z, tr, vel)

    # 4. tiny and ragged: tracePts = 3 (only samples 1 and 2 can be picked), two
    #    traces, negative x step, tau axis reaching past the traces
    tr = np.array([[5.0, -3.0, 2.5], [1.0, 7.0, -4.0]], np.float32)
    run_case(os.path.join(HERE, "ref_tiny.npz"), (3, -7.0, 5.0), (2, 3.0, 1.0),
             (33, 0.0005, 0.0), 0.005, np.array([1.0, 3.0], np.float32),
             np.array([2.0, 0.0], np.float32), np.array([0.5, 2.0], np.float32),
             np.array([-0.25, 1.0], np.float32), tr, np.full(33, 1500.0, np.float32))

    # 5. IBM-32 words -> IEEE through the reference's ktmIBM32toIEEE
    words = np.concatenate([
        rng.integers(0, 2**32, 4000, dtype=np.uint64).astype(np.uint32),
        np.array([0x00000000, 0x80000000, 0x41100000, 0xC1100000, 0x42640000, 0x3F800000,
                  0x7FFFFFFF, 0xFFFFFFFF, 0x00FFFFFF, 0x01000001, 0x7F000000, 0x60FFFFFF,
                  0x20FFFFFF, 0x1F800000], np.uint32)])
    out = oracle.ibm32_to_ieee_reference_c(words)
    np.savez_compressed(os.path.join(HERE, "ref_ibm32.npz"), words=words, ieee=out)
    print("ref_ibm32.npz", words.shape)


if __name__ == "__main__":
    if not oracle.ref_available():
        oracle.build()
    main()
