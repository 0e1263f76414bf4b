"""Build libpcomgpu.so in-tree for sm_100a with nvcc.

The FP64 kernels are compiled with ``--fmad=false`` (no FMA contraction) so
that every operation rounds exactly where the reference's x86-64 build rounds;
the host driver is compiled with ``-ffp-contract=off`` for the same reason.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libpcomgpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FP64 = ["k_step.cu", "k_trop.cu", "pcom_gpu.cu", "k_trop_noalloc.cu", "k_trop_batch.cu"]
# may contract a*b+c into FMA: closure network, mixed barotropic kernels
CU_FAST = ["k_cnn.cu", "cnn.cu", "k_trop_mixed.cu", "k_trop_multi_mixed.cu"]
CPP = ["pcom_host.cpp"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    # /usr/bin/g++ is the system compiler nvcc was validated against
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _sources():
    return [os.path.join(SRC, f) for f in CU_FP64 + CU_FAST + CPP] + [
        os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cuh", ".h"))
    ] + [os.path.join(HERE, "..", "include", f) for f in ("pcom_gpu.h", "pcom_host.h", "pcom_cnn.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in _sources() if os.path.exists(s))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    obj_dir = os.path.join(OUT_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    nvcc = _nvcc()
    cxx = _host_cxx()
    common = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", cxx]
    objs = []
    for f in CU_FP64 + CU_FAST:
        o = os.path.join(obj_dir, f + ".o")
        fmad = ["--fmad=false"] if f in CU_FP64 else ["--fmad=true"]
        cmd = [nvcc, *ARCH, *common, *fmad, "-c", os.path.join(SRC, f), "-o", o]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(o)
    for f in CPP:
        o = os.path.join(obj_dir, f + ".o")
        cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-c", os.path.join(SRC, f), "-o", o]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(o)
    cmd = [nvcc, *ARCH, "-shared", "-ccbin", cxx, "-cudart", "static", "-o", LIB, *objs,
           "-Xlinker", "--exclude-libs,ALL"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
