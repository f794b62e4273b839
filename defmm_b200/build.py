"""Build the CUDA library in-tree: defmm_b200/libdefmm_b200.so (sm_100a).

The library is the product: hand-written CUDA kernels for sm_100a, the host
C++ plan builder and the C ABI declared in include/defmm_b200.h.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdefmm_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU = ["fmm_kernels.cu", "tc_interp.cu", "engine.cu", "noalloc.cu", "plan_device.cu", "near_device.cu", "mlp.cu",
      "measure.cu"]
# the device level walk reproduces the host plan's floating-point decisions:
# no FMA contraction there
CU_FLAGS = {"plan_device.cu": ["--fmad=false"]}
CPP = ["plan.cpp"]
HEADERS = ["plan.hpp", "kernels.cuh", "device_math.cuh", "ptx.cuh", "fp64_math.hpp", "fmm_kernels.h", "engine_internal.h", "plan_device.hpp"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", "defmm_b200.h")]
    objs = []
    jobs = []
    for f in CU:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + hdrs):
            jobs.append([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                         *CU_FLAGS.get(f, []), "-Xptxas", "-v" if verbose else "-O3", "-c", src, "-o", obj])
    for f in CPP:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _newer(obj, [src] + hdrs):
            # discrete results (tree, admissibility, cones) must be the
            # reference's IEEE results: no FMA contraction, no fast-math
            jobs.append(["g++", "-std=c++17", "-O2", "-fPIC", "-pthread", "-ffp-contract=off",
                         "-fno-fast-math", "-c", src, "-o", obj])
    procs = [(j, subprocess.Popen(j, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
             for j in jobs]
    for j, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"build failed: {' '.join(j)}\n{out}")
        if verbose and out:
            print(out, file=sys.stderr)
    if force or jobs or _newer(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lpthread"]
        cp = subprocess.run(cmd, capture_output=True, text=True)
        if cp.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{cp.stdout}{cp.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
