"""Builds librf_b200.so (the C-ABI and every sm_100a kernel) in-tree.

    python -m randomfield_b200.build                 # incremental
    python -m randomfield_b200.build --clean         # from scratch
    python -m randomfield_b200.build --debug-bounds  # librf_b200_bounds.so

The --debug-bounds variant compiles the same sources with -DRF_DEBUG_BOUNDS:
device index checks record a failed check in the context's error word and
skip the access (RF_EBOUNDS), the stand-in for a device memory checker.
Select it at run time with RF_LIB=<path of librf_b200_bounds.so>.

nvcc cross-compiles for sm_100a without a GPU.  Objects go to
randomfield_b200/_build/ (git-ignored), the library next to this file so
that it travels with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librf_b200.so")
BUILD_BOUNDS = os.path.join(HERE, "_build_bounds")
LIB_BOUNDS = os.path.join(HERE, "librf_b200_bounds.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]
SOURCES = ["rf_tables.cu", "rf_tc.cu", "rf_outer.cu", "rf_outer_pair.cu", "rf_fp32.cu", "rf_post.cu", "rf_host.cu", "rf_noalloc.cu", "rf_batch.cu", "rf_serve.cu", "rf_selftest.cu", "rf_stats.cu", "rf_fft.cu", "rf_grid.cu", "rf_writer.cu"]


def _deps(src: str) -> list[str]:
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return [os.path.join(CSRC, src)] + hdrs + [os.path.join(HERE, "..", "include", "randomfield_b200.h")]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, verbose: bool, bounds: bool = False) -> str:
    obj = os.path.join(BUILD_BOUNDS if bounds else BUILD, src.replace(".cu", ".o"))
    if _stale(obj, _deps(src)):
        extra = ["-DRF_DEBUG_BOUNDS"] if bounds else []
        cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
    return obj


def build(clean: bool = False, verbose: bool = False, bounds: bool = False) -> str:
    bdir, lib = (BUILD_BOUNDS, LIB_BOUNDS) if bounds else (BUILD, LIB)
    if clean and os.path.isdir(bdir):
        shutil.rmtree(bdir)
    os.makedirs(bdir, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, bounds), SOURCES))
    if _stale(lib, objs):
        tmp = lib + ".tmp"
        cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/smem usage")
    ap.add_argument("--debug-bounds", action="store_true", help="build librf_b200_bounds.so (-DRF_DEBUG_BOUNDS)")
    a = ap.parse_args()
    print(build(clean=a.clean, verbose=a.verbose, bounds=a.debug_bounds))
