"""Build recipe for libferrox_b200.so and the ferrox_b200 executable.

nvcc compiles the CUDA sources for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``); g++ compiles the host-only sources.  The
outputs land in-tree, next to this file, so they travel with the repository.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libferrox_b200.so")
EXE = os.path.join(HERE, "ferrox_b200")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CU = ["fx_kernels.cu", "fx_mg.cu", "fx_adjoint.cu", "fx_api.cu", "fx_noalloc.cu"]
CPP = ["inputs.cpp", "plotfile.cpp"]
HDR = ["fx_ctl.h", "fx_device.cuh", "fx_kernels.h", "fx_mg.h", "fx_params.h", "plotfile.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-O3"]


def _newer(out: str, deps: list[str]) -> bool:
    return os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HDR] + [os.path.join(HERE, "..", "include", "ferrox_b200.h")]
    objs, jobs = [], []
    for src in CU:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or not _newer(o, [s] + hdrs):
            jobs.append([NVCC] + NVFLAGS + ["-c", s, "-o", o])
        objs.append(o)
    for src in CPP:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or not _newer(o, [s] + hdrs):
            jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", "-c", s, "-o", o])
        objs.append(o)
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, cmd, verbose) for cmd in jobs]:
            f.result()
    if force or not _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lpthread", "-ldl", "-lrt"], verbose)
        os.replace(LIB + ".tmp", LIB)
    main = os.path.join(CSRC, "main.cpp")
    if force or not _newer(EXE, [main, LIB]):
        _run(["g++", "-O2", "-std=c++17", "-o", EXE, main, "-L" + HERE, "-lferrox_b200",
              "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
