"""Build libqsb200.so in-tree: every CUDA source compiled for sm_100a with
nvcc, then linked into one shared library with a static CUDA runtime."""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
OUT = os.path.join(PKG, "libqsb200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
        "-Xptxas", "-warn-spills"]
# Translation units whose arithmetic must follow the reference's expression
# order without FMA contraction (bit-exact FP64 against the oracle).
NO_FMAD = {"push_f64.cu", "spectral.cu", "beam.cu"}
SOURCES = ["api.cu", "dtt_simt.cu", "dtt_tc.cu", "push_f64.cu", "push_f64fma.cu", "push_f32.cu", "spectral.cu",
           "spectral_f32.cu", "beam.cu", "noalloc.cu", "adjoint.cu", "sort.cu", "dtt_fft.cu",
           "pack.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(PKG, "..", "include", "qsb200.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    cmd = [nvcc()] + ARCH + BASE + (["-fmad=false"] if src in NO_FMAD else []) + \
          ["-c", path, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(o) for o in objs):
        return OUT
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", OUT] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
