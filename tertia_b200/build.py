"""Build libqsb200.so in-tree: every CUDA source compiled for sm_100a with
nvcc, then linked into one shared library with a static CUDA runtime.  Beside
it, libqsb200_trace.so: the same library with the march kernels' device
timeline compiled in (csrc/trace.cuh; the units that hold those kernels are
compiled again with -DQS_TRACE, and trace.cu adds qs_trace_attach)."""
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
OUT_TRACE = os.path.join(PKG, "libqsb200_trace.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
        "-Xptxas", "-warn-spills"]
# Translation units whose arithmetic must follow the reference's expression
# order without FMA contraction (bit-exact FP64 against the oracle).
NO_FMAD = {"push_f64.cu", "spectral.cu", "beam.cu"}
SOURCES = ["api.cu", "dtt_simt.cu", "dtt_tc.cu", "push_f64.cu", "push_f64fma.cu", "push_f32.cu", "spectral.cu",
           "spectral_f32.cu", "beam.cu", "noalloc.cu", "adjoint.cu", "sort.cu", "dtt_fft.cu",
           "pack.cu"]
# the units holding instrumented kernels, and the unit only the traced library has
TRACED = ["push_f32.cu", "push_f64fma.cu", "dtt_fft.cu", "sort.cu"]
TRACE_ONLY = ["trace.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: str, verbose: bool, traced: bool = False) -> str:
    out_dir = os.path.join(BUILD, "trace") if traced else BUILD
    obj = os.path.join(out_dir, src.replace(".cu", ".o"))
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps += [os.path.join(PKG, "..", "include", h) for h in ("qsb200.h", "qsb200_trace.h")]
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    cmd = [nvcc()] + ARCH + BASE + (["-fmad=false"] if src in NO_FMAD else []) + \
          (["-DQS_TRACE"] if traced else []) + ["-c", path, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def _link(out: str, objs: list[str]) -> None:
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(o) for o in objs):
        return
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", out] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")


def build(verbose: bool = False) -> str:
    """Build libqsb200.so and libqsb200_trace.so; returns the former's path."""
    os.makedirs(os.path.join(BUILD, "trace"), exist_ok=True)
    jobs = [(s, False) for s in SOURCES] + [(s, True) for s in TRACED + TRACE_ONLY]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda j: _compile(j[0], verbose, j[1]), jobs))
    plain = objs[:len(SOURCES)]
    traced = dict(zip(TRACED + TRACE_ONLY, objs[len(SOURCES):]))
    _link(OUT, plain)
    _link(OUT_TRACE, [traced.get(s, o) for s, o in zip(SOURCES, plain)] +
          [traced[s] for s in TRACE_ONLY])
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
