"""Build the CUDA library in-tree: wrapd_b200/_lib/libwrapd_gpu.so (sm_100a),
and the command-line front end wrapd_b200/_lib/quasi that links it.

Run as ``python -m wrapd_b200.build`` or through ``__graft_entry__.build()``.
Objects are rebuilt only when a source or header is newer than them.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT, "libwrapd_gpu.so")
QUASI = os.path.join(OUT, "quasi")
SOURCES = ["symbolic.cpp", "chol.cu", "solver.cu", "capi.cu", "elem_batch.cu", "prox_net.cu", "dmma_peak.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-lineinfo",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", f"-I{os.path.join(ROOT, 'include')}"]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _deps_mtime() -> float:
    files = glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max(os.path.getmtime(f) for f in files)


def _compile(src: str) -> str:
    obj = os.path.join(OUT, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    if os.path.exists(obj) and os.path.getmtime(obj) >= _deps_mtime():
        return obj
    cmd = [_nvcc(), *NVCC_FLAGS, "-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [_nvcc(), *NVCC_FLAGS, "-x", "c++", "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(_compile, SOURCES))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", LIB]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    quasi_src = os.path.join(CSRC, "quasi.cpp")
    if not os.path.exists(QUASI) or os.path.getmtime(QUASI) < max(os.path.getmtime(LIB), os.path.getmtime(quasi_src)):
        cmd = ["g++", "-O2", "-std=c++17", quasi_src, "-o", QUASI, f"-L{OUT}", "-lwrapd_gpu",
               "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"quasi build failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
