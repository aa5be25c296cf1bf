"""Compiles the reference's DF functions for the host (the reference pin).

TEST INFRASTRUCTURE ONLY. Compiles oracle/ref_pin.cpp with g++, which
#includes src/render/guided/train.cu (and through it train.h, AR.h,
guideditem.h, workqueue.h) unmodified from the reference tree, with
oracle/ref_stub/ as the stand-in framework headers.
Output: oracle/_ref/libgdf_refpin.so (git-ignored; it travels with the tree).
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
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-w",
           "-I", os.path.join(HERE, "ref_stub"), "-I", guided, "-I", os.path.join(ref, "src"),
           "-I", "/usr/local/cuda/include", "-o", SO + ".tmp", *srcs]
    subprocess.run(cmd, check=True)
    os.replace(SO + ".tmp", SO)
    return SO


if __name__ == "__main__":
    print(build("--force" in sys.argv))
