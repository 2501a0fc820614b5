"""Build recipe for the CUDA engine and the C drivers (sm_100a only).

    python ubiquitous-spoon_b200/build.py        # builds in place, next to this file

Produces libchanfast_cuda.so (device engine + cf_* C ABI) and libchanfast.so
(drop-in chanfast2/chanfast4 drivers in C) in this directory.  Device code is
compiled with -fmad=false so that multiply-add sequences round like the
reference CPU build (x86-64, no FMA contraction), except the files listed in
FMA_SOURCES (the substep kernels): contracting a multiply and an add into
one fused operation (one rounding instead of two) cuts their FP64 instruction
count and the latency of their recurrences; results then differ from the
reference by rounding only.  instance.cu keeps -fmad=false: its seeded
initial state must equal the reference's bit for bit.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "nvcc")
CC = os.environ.get("CC", "gcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_SOURCES = ["host_band.cpp", "kernels_rhs.cu", "kernels_solve.cu", "kernels_pressure.cu", "instance.cu",
                "serve.cpp"]
FMA_SOURCES = {"kernels_rhs.cu", "kernels_solve.cu", "kernels_pressure.cu"}
LIB_CUDA = os.path.join(HERE, "libchanfast_cuda.so")
# The reference's step functions (include/chanfast_steps.h): their own
# library, bit-exact arithmetic (no FMA contraction).
STEPS_SOURCE = "steps.cu"
LIB_STEPS = os.path.join(HERE, "libchanfast_steps.so")
LIB_DRIVER = os.path.join(HERE, "libchanfast.so")


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout)
        raise RuntimeError(f"build step failed: {cmd[0]} {os.path.basename(cmd[-1])}")
    return r.stdout


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose=False, ptxas_info=False):
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "chanfast_cuda.h"))
    objs = []
    for src in CUDA_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(objdir, src + ".o")
        objs.append(obj)
        if not _stale(obj, [path] + headers):
            continue
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17",
               "-fmad=true" if src in FMA_SOURCES else "-fmad=false", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-ffp-contract=off", "-I", CSRC, "-I", INCLUDE, "-c", path, "-o", obj]
        if ptxas_info and src.endswith(".cu"):
            cmd[1:1] = ["-Xptxas", "-v"]
        out = _run(cmd)
        if verbose or ptxas_info:
            sys.stdout.write(out)
    if _stale(LIB_CUDA, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB_CUDA, *objs, "-lcudart"])
    steps_src = os.path.join(CSRC, STEPS_SOURCE)
    steps_hdr = os.path.join(INCLUDE, "chanfast_steps.h")
    if os.path.exists(steps_src) and _stale(LIB_STEPS, [steps_src, steps_hdr] + headers):
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--extended-lambda", "-Xcompiler",
               "-fPIC", "-Xcompiler", "-ffp-contract=off", "-I", INCLUDE, "-shared", steps_src, "-o", LIB_STEPS,
               "-Xlinker", "-Bsymbolic", "-lcudart"]
        if ptxas_info:
            cmd[1:1] = ["-Xptxas", "-v"]
        out = _run(cmd)
        if verbose or ptxas_info:
            sys.stdout.write(out)
    drv = os.path.join(CSRC, "chanfast_driver.c")
    if os.path.exists(drv) and _stale(LIB_DRIVER, [drv, LIB_CUDA] + headers):
        _run([CC, "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-I", INCLUDE, drv, "-o", LIB_DRIVER,
              "-L", HERE, "-lchanfast_cuda", "-Wl,-rpath,$ORIGIN", "-lm"])
    return LIB_CUDA


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB_CUDA)
