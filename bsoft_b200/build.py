"""Build libbsgpu.so in-tree with nvcc for sm_100a (no JIT, no torch
extension machinery): ``python -m bsoft_b200.build``."""
from __future__ import annotations

import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build", "libbsgpu.so")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(HERE, "..", "include", "bsgpu.h")]
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


HOSTDIR = os.path.join(HERE, "host")
HOST_PROGRAMS = ("breconstruct", "brefine", "bbackproj")


def build_host(force: bool = False) -> list:
    """The C++ drop-in executables over libbsgpu (bsoft_b200/host)."""
    cxx = shutil.which("g++") or "g++"
    out = []
    for name in HOST_PROGRAMS:
        src = os.path.join(HOSTDIR, name + ".cpp")
        exe = os.path.join(os.path.dirname(OUT), name)
        deps = [src, os.path.join(HOSTDIR, "project.hpp"), OUT, os.path.join(HERE, "..", "include", "bsgpu.h")]
        if force or not os.path.exists(exe) or os.path.getmtime(exe) < max(os.path.getmtime(d) for d in deps):
            tmp = exe + ".tmp"
            subprocess.run([cxx, "-O2", "-std=c++17", "-Wall", "-I", os.path.join(HERE, "..", "include"), src,
                            "-L", os.path.dirname(OUT), "-lbsgpu", "-Wl,-rpath,$ORIGIN", "-o", tmp], check=True)
            os.replace(tmp, exe)
        out.append(exe)
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    if force or not up_to_date():
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        tmp = OUT + ".tmp"
        cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", tmp] + sources()
        subprocess.run(cmd, check=True)
        os.replace(tmp, OUT)
    build_host(force)
    return OUT


if __name__ == "__main__":
    import sys
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
