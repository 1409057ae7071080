"""Builds libamethyst_b200.so in-tree with nvcc for sm_100a.

The library is plain CUDA C++ with a C ABI (include/amethyst.h); nothing here depends on
torch.  Sources are only rebuilt when they are newer than the library.
"""
from __future__ import annotations

import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libamethyst_b200.so")
BUILD_DIR = os.path.join(ROOT, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v"]

UNITS = ["amx_capi.cu", "amx_dispatch.cu", "amx_swar.cu", "amx_swar_w0.cu", "amx_swar_w1.cu", "amx_swar_w2.cu", "amx_swar_w3.cu", "amx_datagen.cu", "amx_noalloc.cu", "amx_groupby.cu", "amx_groupby_sort.cu", "amx_matmul.cu", "amx_mm_fused.cu", "amx_mm_fused_w0.cu", "amx_mm_fused_w1.cu", "amx_batch.cu", "amx_selector.cu", "amx_pairs.cu", "amx_program.cu", "amx_stats.cu"]


def _sources():
    return [os.path.join(CSRC, u) for u in UNITS if os.path.exists(os.path.join(CSRC, u))]


def _deps():
    return glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every translation unit to an object (in parallel) and link the library."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    deps = _deps()
    if not force and not _stale(LIB, deps):
        return LIB
    procs = []
    objs = []
    for src in _sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if not force and not _stale(obj, deps):
            continue
        log = open(obj + ".log", "w")
        cmd = ["nvcc", *FLAGS, *ARCH, "-c", src, "-o", obj]
        procs.append((subprocess.Popen(cmd, stdout=log, stderr=subprocess.STDOUT), cmd, obj + ".log"))
    for p, cmd, logp in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n" + open(logp).read()[-4000:])
    cmd = ["nvcc", *ARCH, "-shared", *objs, "-o", LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
