"""Build libpcomgpu.so in-tree for sm_100a with nvcc.

The step kernels (k_step.cu, k_trop.cu, k_trop_batch.cu) are compiled twice:
with ``--fmad=false`` (no FMA contraction) into namespace ``kx_exact``, so
that every operation rounds exactly where the reference's x86-64 build
rounds, and with ``--fmad=true`` into namespace ``kx_fma`` for handles created
with PCOM_FMA.  The host driver is compiled with ``-ffp-contract=off``.
Objects are compiled in parallel.
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
CU_VARIANT = ["k_step.cu", "k_trop.cu", "k_trop_batch.cu"]  # built exact and contracted
CU_FP64 = ["pcom_gpu.cu", "k_trop_noalloc.cu"]
CU_FAST = ["k_cnn.cu", "cnn.cu", "k_trop_mixed.cu"]  # may contract a*b+c into FMA: closure network, mixed barotropic
CPP = ["pcom_host.cpp"]
VARIANTS = {"exact": ["--fmad=false", "-DPCOM_KNS=kx_exact"], "fma": ["--fmad=true", "-DPCOM_KNS=kx_fma"]}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    # /usr/bin/g++ is the system compiler nvcc was validated against
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _sources():
    return [os.path.join(SRC, f) for f in CU_VARIANT + CU_FP64 + CU_FAST + CPP] + [
        os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cuh", ".h", ".inc"))
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
    jobs = []  # (command, object)
    for f in CU_VARIANT:
        for v, flags in VARIANTS.items():
            o = os.path.join(obj_dir, f"{f}.{v}.o")
            jobs.append(([nvcc, *ARCH, *common, *flags, "-c", os.path.join(SRC, f), "-o", o], o))
    for f in CU_FP64 + CU_FAST:
        o = os.path.join(obj_dir, f + ".o")
        fmad = ["--fmad=false"] if f in CU_FP64 else ["--fmad=true"]
        jobs.append(([nvcc, *ARCH, *common, *fmad, "-c", os.path.join(SRC, f), "-o", o], o))
    for f in CPP:
        o = os.path.join(obj_dir, f + ".o")
        jobs.append(([cxx, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-c", os.path.join(SRC, f), "-o", o], o))
    if verbose:
        for cmd, _ in jobs:
            print(" ".join(cmd))
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda j: subprocess.run(j[0], capture_output=True, text=True), jobs))
    for (cmd, _), r in zip(jobs, results):
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise subprocess.CalledProcessError(r.returncode, cmd)
    objs = [o for _, o in jobs]
    cmd = [nvcc, *ARCH, "-shared", "-ccbin", cxx, "-cudart", "static", "-o", LIB, *objs,
           "-Xlinker", "--exclude-libs,ALL"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
