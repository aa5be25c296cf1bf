"""Builds the guiding module's shared library (libgdf_b200.so) in-tree.

All device code is compiled for sm_100a only. Kernel translation units are
compiled with -fmad=false so the float epilogue keeps the reference's
rounding sequence (explicit fmaf() calls still emit FMAs).

    python guiding-df_b200/build.py [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libgdf_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]

# (source, extra flags)
SOURCES = [
    ("kernels/df_fused.cu", ["-fmad=false"]),
    ("kernels/grid_features.cu", ["-fmad=false"]),
    ("kernels/df_train.cu", ["-fmad=false"]),
    ("kernels/loss_static.cu", []),
    ("kernels/nrc.cu", ["-fmad=false"]),
    ("kernels/paths.cu", ["-fmad=false"]),
    ("kernels/tools.cu", ["-fmad=false"]),
    ("kernels/grouped.cu", ["-fmad=false"]),
    ("host/api.cpp", []),
    ("host/group.cpp", []),
    ("host/serve.cpp", []),
]


def _obj(src: str) -> str:
    return os.path.join(BUILD, src.replace("/", "_") + ".o")


def _deps_mtime() -> float:
    m = 0.0
    for d, _, files in os.walk(CSRC):
        for f in files:
            m = max(m, os.path.getmtime(os.path.join(d, f)))
    m = max(m, os.path.getmtime(os.path.join(ROOT, "include", "gdf.h")))
    return m


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    newest = _deps_mtime()
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB

    def compile_one(item):
        src, extra = item
        obj = _obj(src)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
            return obj
        lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
        cmd = [NVCC, *COMMON, *ARCH, *extra, *lang, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        return obj

    jobs = jobs or min(len(SOURCES), os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs, "-lpthread", "-ldl", "-lrt"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.jobs, a.verbose))
    sys.exit(0)
