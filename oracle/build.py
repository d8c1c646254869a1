"""Build recipe for the CPU oracle (TEST INFRASTRUCTURE ONLY).

Compiles oracle/ofx_oracle.cpp with g++ (OpenMP, FP64, no floating-point
contraction so that x86 and aarch64 hosts round the same way) into
oracle/_build/libofx_oracle.so.  The reference itself cannot be compiled in
this tree: every FerroX source includes AMReX headers and AMReX is absent.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libofx_oracle.so")


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "ofx_oracle.cpp")
    hdr = os.path.join(HERE, "ofx_oracle.h")
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(src), os.path.getmtime(hdr)):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           "-Wall", "-o", LIB + ".tmp", src]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
