"""Compiles the reference's DF functions for the host (the reference pin).

TEST INFRASTRUCTURE ONLY. Compiles oracle/ref_pin.cpp with g++, which
#includes src/render/guided/train.h unmodified from the reference tree at
/root/reference, with oracle/ref_stub/ as the stand-in framework headers.
Output: oracle/_ref/libgdf_refpin.so (git-ignored; it travels with the tree).
No reference source is copied; without /root/reference nothing is built.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("GDF_REFERENCE_ROOT", "/root/reference")
OUT_DIR = os.path.join(HERE, "_ref")
SO = os.path.join(OUT_DIR, "libgdf_refpin.so")


def build(force: bool = False) -> str | None:
    guided = os.path.join(REF, "src", "render", "guided")
    if not os.path.isdir(guided):
        return SO if os.path.exists(SO) else None
    srcs = [os.path.join(HERE, "ref_pin.cpp")]
    deps = srcs + [os.path.join(guided, f) for f in ("train.h", "AR.h", "parameters.h", "guideditem.h",
                                                        "workqueue.h")]
    for d, _, files in os.walk(os.path.join(HERE, "ref_stub")):
        deps += [os.path.join(d, f) for f in files]
    if not force and os.path.exists(SO) and os.path.getmtime(SO) >= max(os.path.getmtime(p) for p in deps):
        return SO
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-w",
           "-I", os.path.join(HERE, "ref_stub"), "-I", guided, "-I", os.path.join(REF, "src"),
           "-I", "/usr/local/cuda/include", "-o", SO + ".tmp", *srcs]
    subprocess.run(cmd, check=True)
    os.replace(SO + ".tmp", SO)
    return SO


if __name__ == "__main__":
    print(build("--force" in sys.argv))
