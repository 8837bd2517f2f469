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
