"""Build the engine in-tree: libfastgrid_b200.so (CUDA kernels for sm_100a,
the C ABI and the C++ host code) and the fastgrid4 / autogrid4 executables.

    python -m fastgrid_b200.build          # or fastgrid_b200.build.build()

nvcc cross-compiles for sm_100a without a GPU.  Host C++ is compiled with
-ffp-contract=off so its double arithmetic rounds like the reference's.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
OBJ = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU = ["emap.cu", "affinity.cu", "affinity2.cu", "cells.cu", "capi.cu", "peaks.cu", "emap_noalloc.cu", "surrogate.cu",
      "surrogate_host.cu", "surr_near.cu", "surr_tc.cu"]
CPP = ["host.cpp", "synth.cpp"]
LIB = os.path.join(OUT, "libfastgrid_b200.so")


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r.stdout


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose=False, ptxas_v=False):
    os.makedirs(OUT, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "fastgrid_b200.h"))
    objs = []
    for f in CU:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            cmd = [NVCC] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                                   "-c", "-o", obj, src]
            if ptxas_v:
                cmd.insert(1, "-Xptxas=-v")
            out = _run(cmd)
            if verbose or ptxas_v:
                sys.stdout.write(out)
    for f in CPP:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-c", "-o", obj, src])
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"])
    exe = os.path.join(OUT, "fastgrid4")
    main = os.path.join(CSRC, "cli_main.cpp")
    if _stale(exe, [main, LIB]):
        _run(["g++", "-O2", "-o", exe, main, "-L" + OUT, "-lfastgrid_b200", "-Wl,-rpath,$ORIGIN"])
    ag4 = os.path.join(OUT, "autogrid4")
    if _stale(ag4, [exe]):
        shutil.copy2(exe, ag4)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_v="-v" in sys.argv)
    print(LIB)
