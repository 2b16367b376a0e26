"""Build liblbm_b200.so in-tree with nvcc for sm_100a.

The kernel source is compiled twice: once for the fast arithmetic mode and
once, with --fmad=false and LBM_EXACT=1, for the exact mode that reproduces the
reference's FP64 operation order.  Host code is compiled without multiply-add
contraction so derived parameters and interpolation weights match the
reference's arithmetic.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "liblbm_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


UNITS = [
    # (object, source, extra flags)
    ("kernels_fast.o", "lbm_kernels.cu", ["-DLBM_NS=fast"]),
    ("kernels_exact.o", "lbm_kernels.cu", ["-DLBM_NS=exact", "-DLBM_EXACT=1", "--fmad=false"]),
    ("reduce.o", "lbm_reduce.cu", ["--fmad=false"]),
    ("capi.o", "lbm_capi.cu", []),
    ("noalloc.o", "lbm_noalloc.cu", ["--fmad=false"]),
    ("batch.o", "lbm_batch.cu", []),
    ("unet.o", "unet_kernels.cu", []),
]

HEADERS = ["lbm_internal.h", "lbm_handle.h", "lbm_march.cuh"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", h)
                                                        for h in ("lbm_b200.h", "lbm_surrogate.h")]
    objs = []
    for obj, src, extra in UNITS:
        o = os.path.join(BUILD, obj)
        s = os.path.join(CSRC, src)
        objs.append(o)
        if force or ptxas_info or _stale(o, [s, __file__] + hdrs):
            cmd = [cc, *ARCH, *COMMON, *extra, "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.check_call(cmd)
    if force or _stale(LIB, objs):
        cmd = [cc, *ARCH, "-shared", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
