"""Build libktm.so (sm_100a) and the psktm command-line driver in-tree.

    python seismic-migration_b200/build.py [--force] [--jobs N]

Every .cu file under csrc/ is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into
``ktm/_build/*.o`` and linked into ``ktm/libktm.so``; C sources of the host
side are compiled with gcc.  Objects are rebuilt only when a source or a
header is newer.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
PKG = os.path.join(HERE, "ktm")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libktm.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
                  "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-I" + INCLUDE]


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    csrcs = sorted(glob.glob(os.path.join(CSRC, "*.c")))
    objs, work = [], []
    for s in srcs + csrcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            if s.endswith(".cu"):
                cmd = [NVCC] + NVFLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", s, "-o", o]
            else:
                cmd = ["gcc", "-O2", "-fPIC", "-ffp-contract=off", "-std=c11", "-I" + INCLUDE,
                       "-c", s, "-o", o]
            work.append(cmd)
    log = []
    if work:
        with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
            for out in ex.map(_run, work):
                log.append(out)
    if force or work or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs)
    drv_src = os.path.join(HERE, "psktm.c")
    drv = os.path.join(PKG, "psktm")
    if os.path.exists(drv_src) and (force or _stale(drv, [drv_src, LIB] + headers)):
        _run(["gcc", "-O2", "-std=c11", "-I" + INCLUDE, drv_src, "-o", drv,
              "-L" + PKG, "-lktm", "-Wl,-rpath,$ORIGIN"])
    return "\n".join(log)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    out = build(a.force, a.jobs, a.verbose)
    if a.verbose:
        print(out)
    print("built", LIB)
