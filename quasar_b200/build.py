"""Build the sm_100a extension in-tree: quasar_b200/_lib/libquasar_mhd_b200.so.

    python -m quasar_b200.build          # incremental (per-object mtime)
    python -m quasar_b200.build --force

nvcc cross-compiles for sm_100a without a GPU.  Objects go to
quasar_b200/_build/ (git-ignored); the shared library is git-ignored but
travels with the repository snapshot.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libquasar_mhd_b200.so")
SOURCES = ["mhd_kernels.cu", "mhd_solver.cu", "mhd_batch.cu", "capi.cu", "probe.cu", "noalloc.cu", "indicator.cu", "launch_abi.cu"]
HEADERS = ["mhd_device.cuh", "mhd_kernels.cuh", "mhd_solver.cuh", "mhd_batch.cuh", "noalloc.cuh", "indicator.cuh", "tc.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-diag-suppress", "177"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def _compile(src: str, force: bool, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS]
    deps.append(os.path.join(ROOT, "include", "quasar_mhd.h"))
    deps.append(os.path.join(ROOT, "include", "quasar_mhd_ext.h"))
    deps.append(os.path.join(ROOT, "include", "quasar_mhd_launch.h"))
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= _newest(deps):
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    with cf.ThreadPoolExecutor(len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), SOURCES))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart=static", "-o", LIB, *objs]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
