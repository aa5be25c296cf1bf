"""Builds the reference's own GPU path for the B200 (the reference GPU harness).

TEST INFRASTRUCTURE ONLY: the product never links or loads what this builds.
Compiles, with nvcc for sm_100a and straight from the reference tree (the
sources are read where they lie; nothing is copied into this repository):
  - tiny-cuda-nn v1.6, vendored at src/ext/tcnn: src/{common, common_device,
    cutlass_mlp, encoding, fully_fused_mlp, loss, network, object, optimizer,
    reduce_sum}.cu with its vendored CUTLASS 2.9 and fmt headers, the flags of
    tcnn/CMakeLists.txt (C++17, --extended-lambda, --expt-relaxed-constexpr,
    TCNN_MIN_GPU_ARCH=90: the newest architecture its CMake accepts, which
    it would pick on a B200) and fmt's format.cc / os.cc, in the Release
    configuration the reference is built in (-O3 -DNDEBUG: its device-side
    assert(mIsTwoSided) in AR.h:33 is compiled out, as in the reference's
    own build, so a record whose fp16 pdf underflows to zero trains on);
  - oracle/ref_gpu/harness.cu, which includes the reference's unmodified
    src/render/guided/train.cu (and through it train.h, AR.h, guideditem.h,
    workqueue.h), once per bin configuration.
The reference fixes its bin counts in parameters.h. For each configuration a
directory of symbolic links under oracle/_ref/shadow/ presents the reference
files together with oracle/ref_gpu/parameters_shadow.h as parameters.h, and
the bin counts come in as -DGDF_REF_BINS_THETA / -DGDF_REF_BINS_PHI.
Outputs (git-ignored, they travel with the tree to the GPU box):
  oracle/_ref/libgdf_tcnnref_<theta>x<phi>.so  for (16, 32), (32, 32), (64, 64)
The reference tree is GDF_REFERENCE_ROOT, or a checkout named `reference`
beside this repository; without one nothing is built and the libraries
built earlier are used.

    python oracle/build_ref_gpu.py [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "tcnn_obj_release")
SHADOW = os.path.join(OUT, "shadow")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BIN_CONFIGS = [(16, 32), (32, 32), (64, 64)]
TCNN_UNITS = ["common", "common_device", "cutlass_mlp", "encoding", "fully_fused_mlp", "loss", "network",
              "object", "optimizer", "reduce_sum"]
GUIDED_FILES = ["train.cu", "train.h", "AR.h", "guideditem.h", "workqueue.h"]


def reference_root() -> str | None:
    """GDF_REFERENCE_ROOT, else ../reference beside the repository."""
    for cand in (os.environ.get("GDF_REFERENCE_ROOT"), os.path.join(os.path.dirname(HERE), os.pardir, "reference")):
        if cand and os.path.isdir(os.path.join(cand, "src", "ext", "tcnn")):
            return os.path.abspath(cand)
    return None


def lib_path(theta: int, phi: int) -> str:
    return os.path.join(OUT, f"libgdf_tcnnref_{theta}x{phi}.so")


def _tcnn_flags(ref: str) -> list[str]:
    t = os.path.join(ref, "src", "ext", "tcnn")
    return ["-std=c++17", "-O3", "-DNDEBUG", "--extended-lambda", "--expt-relaxed-constexpr", "-DTCNN_MIN_GPU_ARCH=90",
            "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-strict-aliasing", "-Xcompiler", "-mf16c", "-w",
            "-Xcudafe", "--diag_suppress=unrecognized_gcc_pragma",
            "-I", os.path.join(t, "include"), "-I", os.path.join(t, "dependencies"),
            "-I", os.path.join(t, "dependencies", "cutlass", "include"),
            "-I", os.path.join(t, "dependencies", "cutlass", "tools", "util", "include"),
            "-I", os.path.join(t, "dependencies", "fmt", "include")]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"failed: {' '.join(cmd)}\n{r.stdout[-4000:]}\n{r.stderr[-4000:]}")


def _shadow(ref: str) -> str:
    """Directory of links: the reference's guided files beside our parameters.h."""
    d = os.path.join(SHADOW, "render", "guided")
    os.makedirs(d, exist_ok=True)
    links = {f: os.path.join(ref, "src", "render", "guided", f) for f in GUIDED_FILES}
    links["parameters.h"] = os.path.join(HERE, "ref_gpu", "parameters_shadow.h")
    for name, target in links.items():
        p = os.path.join(d, name)
        if os.path.islink(p) and os.readlink(p) == target:
            continue
        if os.path.lexists(p):
            os.remove(p)
        os.symlink(target, p)
    return d


def build(force: bool = False, jobs: int = 0) -> list[str]:
    ref = reference_root()
    if ref is None:
        return [p for p in (lib_path(*c) for c in BIN_CONFIGS) if os.path.exists(p)]
    os.makedirs(OBJ, exist_ok=True)
    t = os.path.join(ref, "src", "ext", "tcnn")
    flags = _tcnn_flags(ref)

    def tcnn_unit(name: str) -> str:
        o = os.path.join(OBJ, name + ".o")
        if force or not os.path.exists(o):
            _run([NVCC, *flags, *ARCH, "-c", os.path.join(t, "src", name + ".cu"), "-o", o])
        return o

    def fmt_unit(name: str) -> str:
        o = os.path.join(OBJ, "fmt_" + name + ".o")
        if force or not os.path.exists(o):
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-w", "-I", os.path.join(t, "dependencies", "fmt", "include"),
                  "-c", os.path.join(t, "dependencies", "fmt", "src", name + ".cc"), "-o", o])
        return o

    guided = _shadow(ref)
    harness = os.path.join(HERE, "ref_gpu", "harness.cu")
    stub = os.path.join(HERE, "ref_stub")
    deps = [harness, os.path.join(HERE, "ref_gpu", "parameters_shadow.h")]
    for d, _, files in os.walk(stub):
        deps += [os.path.join(d, f) for f in files]
    newest = max(os.path.getmtime(p) for p in deps)

    def harness_unit(cfg: tuple[int, int]) -> str:
        o = os.path.join(OBJ, f"harness_{cfg[0]}x{cfg[1]}.o")
        if force or not os.path.exists(o) or os.path.getmtime(o) < newest:
            _run([NVCC, *flags, *ARCH, f"-DGDF_REF_BINS_THETA={cfg[0]}", f"-DGDF_REF_BINS_PHI={cfg[1]}",
                  "-I", guided, "-I", SHADOW, "-I", stub, "-c", harness, "-o", o])
        return o

    jobs = jobs or max(1, os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        f_tcnn = [ex.submit(tcnn_unit, u) for u in TCNN_UNITS]
        f_fmt = [ex.submit(fmt_unit, u) for u in ("format", "os")]
        f_h = [ex.submit(harness_unit, c) for c in BIN_CONFIGS]
        common = [f.result() for f in f_tcnn + f_fmt]
        harness_objs = [f.result() for f in f_h]

    out = []
    for cfg, ho in zip(BIN_CONFIGS, harness_objs):
        so = lib_path(*cfg)
        if force or not os.path.exists(so) or os.path.getmtime(so) < max(os.path.getmtime(p) for p in [ho, *common]):
            _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-Xlinker", "-Bsymbolic", "-o", so + ".tmp",
                  ho, *common, "-lcuda", "-lcublas"])
            os.replace(so + ".tmp", so)
        out.append(so)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    a = ap.parse_args()
    if reference_root() is None:
        sys.exit("no reference tree: set GDF_REFERENCE_ROOT")
    for p in build(a.force, a.jobs):
        print(p)
