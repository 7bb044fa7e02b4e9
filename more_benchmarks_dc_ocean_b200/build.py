"""Build the sm_100a shared library (libredi_b200.so) in-tree with nvcc.

The kernels (redi_plain.cu, redi_domains.cu, meke.cu, ale.cu) are compiled with FMA contraction off so their
arithmetic is the reference's IEEE sequence; everything is compiled for
sm_100a only (`-gencode arch=compute_100a,code=sm_100a`).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libredi_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", CSRC, "-I", INCLUDE] + ARCH

# (source, extra flags)
SOURCES = [
    ("redi_plain.cu", ["-fmad=false"]),
    ("redi_capi.cu", []),
    ("redi_noalloc.cu", []),
    ("redi_halo.cu", []),
    ("redi_domains.cu", ["-fmad=false"]),
    ("meke.cu", ["-fmad=false"]),
    ("ale.cu", ["-fmad=false"]),
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the B200 kernels cannot be built")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile every CUDA source and link libredi_b200.so; returns its path."""
    nvcc = _nvcc()
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(INCLUDE, h) for h in ("redi_b200.h", "meke_b200.h", "ale_b200.h")]
    objs = []
    for src, flags in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src.replace(".cu", ".o"))
        objs.append(obj)
        if _stale(obj, [path, __file__] + headers):
            cmd = [nvcc] + COMMON + flags + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if _stale(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
