"""Build recipe of libppf.so (sm_100a), in-tree next to this file.

Runs nvcc directly: one object per .cu file, linked into a shared library
with a plain C ABI (include/ppf.h).  Usable without a GPU (cross-compiles).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libppf.so")
CXX_OUT = os.path.join(HERE, "libppf_cxx.so")   # the C++ driver's solve calls on libppf
BUILD = os.path.join(HERE, "_build")
SOURCES = ["ppf_x.cu", "ppf_y.cu", "ppf_tdma.cu", "ppf_ghost.cu", "ppf_adjoint.cu", "ppf_slab.cu", "ppf_batch.cu", "ppf_post.cu", "ppf_api.cu"]
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, jobs: int = 4) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "ppf.h"))
    objs, procs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + headers):
            cmd = [NVCC, *FLAGS, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
            if len(procs) >= jobs:
                _wait(procs)
    _wait(procs)
    if _stale(OUT, objs):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    build_cxx_driver(verbose)
    return OUT


def build_cxx_driver(verbose: bool = False) -> str:
    """libppf_cxx.so: mpi_poisson::mpi_Poisson_FFT{1..5} of the C++ driver on
    libppf (g++; found next to libppf.so through its run path).  Its
    references to the driver's globals are resolved when the driver's
    program (or a test harness defining them) loads it."""
    src = os.path.join(CSRC, "ppf_cxx_driver.cpp")
    hdrs = [os.path.join(HERE, "..", "include", h) for h in ("ppf.h", "ppf_cxx_driver.h")]
    if _stale(CXX_OUT, [src, OUT] + hdrs):
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
               "-fvisibility=hidden", "-Wall", "-o", CXX_OUT, src, f"-L{HERE}", "-l:libppf.so",
               "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return CXX_OUT


def _wait(procs):
    err = None
    for name, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            err = f"nvcc failed on {name}:\n{text}"
        elif text.strip():
            sys.stderr.write(text)
    procs.clear()
    if err:
        raise RuntimeError(err)


if __name__ == "__main__":
    print(build(verbose=True))
