"""Compiles the reference's DF functions for the host (the reference pin).

TEST INFRASTRUCTURE ONLY. Compiles oracle/ref_pin.cpp with g++, which
#includes src/render/guided/train.cu (and through it train.h, AR.h,
guideditem.h, workqueue.h) unmodified from the reference tree, with
oracle/ref_stub/ as the stand-in framework headers.
Output: oracle/_ref/libgdf_refpin.so (git-ignored; it travels with the tree).
build_cpu_baseline() compiles oracle/ref_cpu.cpp (the reference's
thetaPostInference / phiPostInference for the host, fed by the C oracle's
fp32 forward) per bin configuration into oracle/_ref/libgdf_refcpu_<t>x<p>.so:
the CPU baseline bench.py times.
No reference source is copied. The reference tree is GDF_REFERENCE_ROOT, or
a checkout named `reference` beside this repository; without one nothing is
built and a library built earlier is used.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def reference_root() -> str | None:
    """GDF_REFERENCE_ROOT, else ../reference beside the repository."""
    for cand in (os.environ.get("GDF_REFERENCE_ROOT"), os.path.join(ROOT, os.pardir, "reference")):
        if cand and os.path.isdir(os.path.join(cand, "src", "render", "guided")):
            return os.path.abspath(cand)
    return None


OUT_DIR = os.path.join(HERE, "_ref")
SO = os.path.join(OUT_DIR, "libgdf_refpin.so")


def build(force: bool = False) -> str | None:
    ref = reference_root()
    if ref is None:
        return SO if os.path.exists(SO) else None
    guided = os.path.join(ref, "src", "render", "guided")
    srcs = [os.path.join(HERE, "ref_pin.cpp")]
    deps = srcs + [os.path.join(guided, f) for f in ("train.cu", "train.h", "AR.h", "parameters.h",
                                                        "guideditem.h", "workqueue.h")]
    for d, _, files in os.walk(os.path.join(HERE, "ref_stub")):
        deps += [os.path.join(d, f) for f in files]
    if not force and os.path.exists(SO) and os.path.getmtime(SO) >= max(os.path.getmtime(p) for p in deps):
        return SO
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-DNDEBUG", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-w",
           "-I", os.path.join(HERE, "ref_stub"), "-I", guided, "-I", os.path.join(ref, "src"),
           "-I", "/usr/local/cuda/include", "-o", SO + ".tmp", *srcs]
    subprocess.run(cmd, check=True)
    os.replace(SO + ".tmp", SO)
    return SO


CPU_BIN_CONFIGS = [(32, 32), (64, 64)]


def cpu_lib_path(theta: int, phi: int) -> str:
    return os.path.join(OUT_DIR, f"libgdf_refcpu_{theta}x{phi}.so")


def build_cpu_baseline(force: bool = False) -> list[str]:
    ref = reference_root()
    if ref is None:
        return [p for p in (cpu_lib_path(*c) for c in CPU_BIN_CONFIGS) if os.path.exists(p)]
    import importlib.util
    spec = importlib.util.spec_from_file_location("build_ref_gpu", os.path.join(HERE, "build_ref_gpu.py"))
    gpu = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gpu)
    guided = gpu._shadow(ref)  # the reference files beside parameters_shadow.h
    srcs = [os.path.join(HERE, f) for f in ("ref_cpu.cpp", "gdf_oracle.c")]
    deps = srcs + [os.path.join(HERE, "gdf_oracle.h"), os.path.join(HERE, "ref_gpu", "parameters_shadow.h"),
                   os.path.abspath(__file__)]
    deps += [os.path.join(guided, f) for f in os.listdir(guided)]
    for d, _, files in os.walk(os.path.join(HERE, "ref_stub")):
        deps += [os.path.join(d, f) for f in files]
    newest = max(os.path.getmtime(p) for p in deps)
    out = []
    os.makedirs(OUT_DIR, exist_ok=True)
    for t, p in CPU_BIN_CONFIGS:
        so = cpu_lib_path(t, p)
        if force or not os.path.exists(so) or os.path.getmtime(so) < newest:
            # a portable x86-64 server ISA (the GPU box's host CPU is not this
            # one); no contraction, so the forward equals the oracle's fp32 one
            flags = ["-O3", "-DNDEBUG", "-mavx2", "-mfma", "-ffp-contract=off", "-fopenmp", "-fPIC", "-w"]
            obj = so + ".oracle.o"
            subprocess.run(["gcc", "-std=c11", *flags, "-c", srcs[1], "-o", obj], check=True)
            subprocess.run(["g++", "-std=c++17", *flags, "-shared", f"-DGDF_REF_BINS_THETA={t}",
                            f"-DGDF_REF_BINS_PHI={p}", "-I", guided, "-I", gpu.SHADOW,
                            "-I", os.path.join(HERE, "ref_stub"), "-I", HERE, "-I", "/usr/local/cuda/include",
                            "-o", so + ".tmp", srcs[0], obj], check=True)
            os.remove(obj)
            os.replace(so + ".tmp", so)
        out.append(so)
    return out


if __name__ == "__main__":
    print(build("--force" in sys.argv))
    print(build_cpu_baseline("--force" in sys.argv))
