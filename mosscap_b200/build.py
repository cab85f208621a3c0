"""Build ``mosscap_b200/libmosscap_b200.so`` from ``mosscap_b200/csrc`` for sm_100a.

Every translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo``. The FP64 stage
kernels and the utility kernels are compiled with ``-fmad=false`` so that no
multiply-add is contracted: their results are bit-identical to the
reference's CPU build. The FP32-form kernels use ``--use_fast_math``
(contraction, approximate FP32 division and square root).

Objects go to ``mosscap_b200/_build`` and are rebuilt when any source or
header is newer. Run ``python -m mosscap_b200.build``.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmosscap_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC,
          "--expt-relaxed-constexpr"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _flags_for(src: str) -> list:
    name = os.path.basename(src)
    if "_fp32" in name:
        # the FP32 compute form is not bit-exact by design: approximate FP32
        # division / square root and contraction (FP64 division stays IEEE)
        return ["--use_fast_math"]
    if "_fma" in name:
        # arithmetic that need not be bit-exact (the adjoint's reverse sweep)
        return ["-fmad=true"]
    return ["-fmad=false"]


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max(os.path.getmtime(h) for h in hs) if hs else 0.0


def _compile(src: str, hdr_mtime: float, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
        return obj
    cmd = [nvcc()] + ARCH + COMMON + _flags_for(src) + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, jobs: int = 0) -> str:
    """Compile every kernel source and link the shared library; return its path."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = _headers_mtime()
    jobs = jobs or max(1, min(len(srcs), os.cpu_count() or 1))
    # the biggest translation units first
    srcs.sort(key=lambda s: ("_d3_" not in s, "_d2_" not in s, "_src" in s, s))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, hdr, verbose), srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-ldl"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
