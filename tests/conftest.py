"""Shared test set-up: import paths, the ``gpu`` marker, golden fixtures."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "seismic-migration_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


def golden_grids(g: dict):
    import oracle
    return tuple(oracle.grid(int(a[0]), float(a[1]), float(a[2])) for a in (g["gx"], g["gy"], g["gz"]))


def degenerate_reference_case(seed: int = 44):
    """Reference-mode inputs with degenerate values (host-made, no device fault): a Vrms
    of 0, a negative one, 1e30, +inf and NaN at single tau samples, and +-inf trace
    samples.  psktmCPU.c's float arithmetic turns them into NaN / inf traveltimes (picks
    it skips) and NaN / inf image samples, which reference mode must reproduce."""
    import oracle
    rng = np.random.default_rng(seed)
    ntr, nt, nz = 30, 120, 90
    gx, gy, gz = oracle.grid(5, 30.0, -60.0), oracle.grid(3, 25.0, -20.0), oracle.grid(nz, 0.002, 0.0)
    mid = rng.uniform(-300, 300, (ntr, 2)).astype(np.float32)
    off = rng.uniform(-300, 300, (ntr, 2)).astype(np.float32)
    tr = rng.standard_normal((ntr, nt)).astype(np.float32)
    tr[3, 60:70] = np.inf
    tr[9, 80] = -np.inf
    vel = np.linspace(1500.0, 3000.0, nz).astype(np.float32)
    vel[5], vel[17], vel[40], vel[60], vel[70] = 0.0, -2000.0, 1e30, np.inf, np.nan
    return gx, gy, gz, 0.004, mid[:, 0].copy(), mid[:, 1].copy(), off[:, 0].copy(), off[:, 1].copy(), tr, vel


def same_with_nans(a, b) -> bool:
    """NaN at the same samples (any payload), every other sample bit-identical."""
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    na, nb = np.isnan(a), np.isnan(b)
    return bool(np.array_equal(na, nb) and np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32)))


GOLDEN_MIGRATIONS = ["ref_line_small.npz", "ref_areal_small.npz", "ref_zero_offset.npz",
                     "ref_tiny.npz"]


@pytest.fixture(scope="session")
def ktm_lib():
    """libktm.so, built in-tree if it is missing (nvcc cross-compiles here)."""
    import ktm
    if not os.path.exists(ktm.LIB_PATH):
        sys.path.insert(0, PKG)
        import build  # seismic-migration_b200/build.py
        build.build()
    return ktm.lib()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
