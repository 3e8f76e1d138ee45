"""Build recipe for libplamatrix_b200.so (sm_100a only).

Every translation unit in csrc/ is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a`` and linked into one in-tree shared
library (``plamatrix_b200/_lib/libplamatrix_b200.so``) so that it travels with the
repository snapshot.  Objects are rebuilt only when a source or header changed.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libplamatrix_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
         "-ccbin", "/usr/bin/g++"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, extra) -> str:
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    if _stale(obj, [src, __file__] + _headers()):
        cmd = [NVCC] + ARCH + FLAGS + list(extra) + ["-c", src, "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError(f"nvcc failed for {os.path.basename(src)}")
        if res.stderr.strip():
            sys.stderr.write(res.stderr)
    return obj


def build(verbose: bool = False, extra=()) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    sources = _sources()
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as pool:
        objects = list(pool.map(lambda s: _compile(s, extra), sources))
    if _stale(LIB, objects):
        cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++", "-o", LIB] + objects + \
            ["-lcuda"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("link failed")
    if verbose:
        print(LIB)
    return LIB


def resource_usage(src: str) -> str:
    """ptxas register / spill / shared-memory report of one translation unit."""
    cmd = [NVCC] + ARCH + FLAGS + ["-Xptxas", "-v", "-c", src, "-o", os.devnull]
    res = subprocess.run(cmd, capture_output=True, text=True)
    return res.stdout + res.stderr


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--ptxas":
        for s in sys.argv[2:] or _sources():
            print(resource_usage(s))
    else:
        build(verbose=True)
