"""Build step for libsailfish_b200.so (nvcc, sm_100a), in tree next to this file.

    python -m sailfish_b200.build          # or: python sailfish_b200/build.py

Translation units (sailfish_b200/csrc):
    sf_kernels_f64.cu   FP64 kernels, -fmad=false (IEEE evaluation as written, the parity path)
    sf_kernels_f32.cu   FP32 kernels, FMA contraction on
    sf_capi.cu          C ABI (include/sailfish_b200.h), contexts, boundary programs
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsailfish_b200.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr"]
UNITS = {
    "sf_kernels_f64.cu": ["-fmad=false"],
    "sf_kernels_f32.cu": [],
    "sf_capi.cu": [],
    "sf_mlp.cu": [],
}


def _sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "sailfish_b200.h"), os.path.abspath(__file__)]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in _sources())


def build(verbose=False, force=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for unit, extra in UNITS.items():
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        cmd = [NVCC] + ARCH + COMMON + extra + ["-c", os.path.join(CSRC, unit), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        objs.append(obj)
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
