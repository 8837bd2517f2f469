"""ktm -- B200 prestack Kirchhoff time migration (PSTM), Python host side.

The compute lives in ``libktm.so`` (hand-written sm_100a CUDA behind the C ABI
of include/ktm.h); this package binds it with ctypes, mirrors the reference's
entry points (``ktmMigrationCPU`` and friends) and generates the seeded
synthetic surveys used by the tests and the benchmark.
"""
from ._lib import KtmError, ImageGrid, JobParams, lib, LIB_PATH  # noqa: F401
from .api import (  # noqa: F401
    grid, ktmMigrationCPU, ktmMigrationGPU, initThreeAxes, migrate, migrate_columns_f64, Job,
)
from .api import PackedTraces, packed_pitch, prepare  # noqa: F401,E402
from .api import autotune, autotune_tile, tile_candidates, migrate_batch, interp_time  # noqa: F401,E402
from . import io  # noqa: F401,E402
