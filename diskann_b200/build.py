"""Build recipe of the CUDA library (nvcc, sm_100a only).

``build()`` compiles every ``csrc/*.cu`` (device code and the C ABI) and ``csrc/*.cpp`` (host
code) in parallel into ``_build/`` and links ``_lib/libdiskann_b200.so``.  Objects are rebuilt
only when a source or header is newer than them.
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
CSRC = os.path.join(_HERE, "csrc")
BUILD = os.path.join(_HERE, "_build")
OUT = os.path.join(_HERE, "_lib", "libdiskann_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: no implicit multiply-add contraction; every FMA in the kernels is an explicit
# __fmaf_rn restating a reference FMA, so float results match the reference bit for bit.
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-O2", "-I", os.path.join(_ROOT, "include"), "-I", CSRC,
]
# x86-64-v3 (AVX2 + FMA) like the reference's own target; no contraction beyond explicit fma.
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-pthread", "-mavx2", "-mfma", "-ffp-contract=off", "-I", os.path.join(_ROOT, "include"),
             "-I", CSRC, "-I", "/usr/local/cuda/include"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, headers) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if _newer(obj, [src] + headers):
        if src.endswith(".cu"):
            cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
        else:
            cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
                     + glob.glob(os.path.join(_ROOT, "include", "*.h")))
    with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, headers), sources))
    if _newer(OUT, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(OUT)
    return OUT


if __name__ == "__main__":
    build(verbose=True)
