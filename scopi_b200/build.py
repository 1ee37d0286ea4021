"""Build libscopi_gpu.so (sm_100a) in-tree with nvcc.

detect.cu is compiled with -fmad=false so the closest-point arithmetic keeps the
reference's operation order (the contact set is decided by a strict dij < dmax);
the solver kernels keep FMA contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libscopi_gpu.so")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "--expt-relaxed-constexpr"]
SOURCES = {
    "detect.cu": ["-fmad=false"],
    "apgd.cu": [],
    "apgd_sph.cu": [],
    "apgd_batch.cu": [],
    "se.cu": ["-fmad=false"],
    "scan.cu": [],
    "scopi_gpu.cu": [],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "scopi_gpu.h"),
                                                                 os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, force: bool = False, extra: list | None = None) -> str:
    if not force and not needs_build():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    objs, procs = [], []
    # the translation units are independent: compile them side by side
    for src, flags in SOURCES.items():
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, *COMMON, *flags, *(extra or []), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [cmd for cmd, pr in procs if pr.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    cmd = [nvcc(), *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, extra=[a for a in sys.argv[1:] if a != "--force"])
