"""Build libpevsl_b200.so in-tree (pevsl_b200/libpevsl_b200.so).

Host C modules are compiled with gcc, CUDA modules with nvcc for sm_100a
only, and the library is linked by nvcc (static CUDA runtime).  Objects go to
pevsl_b200/_build/; a module is rebuilt when it or any header is newer than
its object.

    python -m pevsl_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpevsl_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CC = os.environ.get("CC", "gcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O2", "-g", "-std=gnu11", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter",
          "-I" + INC, "-I" + CSRC]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
           "-Xptxas", "-O3", "-I" + INC, "-I" + CSRC] + ARCH


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INC, "*.h"))


def _stale(obj, src, hdr_mtime):
    if not os.path.exists(obj):
        return True
    m = os.path.getmtime(obj)
    return os.path.getmtime(src) > m or hdr_mtime > m


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False, extra_nvflags=None) -> str:
    """Compile the stale modules (in parallel, one process per module) and
    link the library when anything changed."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OUT_DIR, exist_ok=True)
    hdr = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    objs, jobs = [], []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.c"))):
        obj = os.path.join(OUT_DIR, os.path.basename(src) + ".o")
        if force or _stale(obj, src, hdr):
            jobs.append([CC] + CFLAGS + ["-c", src, "-o", obj])
        objs.append(obj)
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(OUT_DIR, os.path.basename(src) + ".o")
        if force or _stale(obj, src, hdr):
            jobs.append([NVCC] + NVFLAGS + (extra_nvflags or []) + ["-c", src, "-o", obj])
        objs.append(obj)
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
            for f in [ex.submit(_run, cmd, verbose) for cmd in jobs]:
                f.result()
    if jobs or force or not os.path.exists(LIB):
        _run([NVCC, "-shared"] + ARCH + ["-o", LIB] + objs + ["-lm"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
