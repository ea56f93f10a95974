"""Builds libnbgpu.so in-tree (nativebigint.jl_b200/lib/libnbgpu.so).

Device code is compiled for sm_100a only, with -fmad=false so nvcc never
contracts a*b+c (the kernels also use explicit _rn intrinsics); host code is
compiled with -ffp-contract=off for the same reason.  Run as a script or
call build().
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc") if os.path.exists(os.path.join(CUDA, "bin", "nvcc")) else "nvcc"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wextra",
             "-Wno-unused-parameter", f"-I{CUDA}/include"]

CU_SOURCES = ["kernels.cu", "noalloc.cu", "powmod_kernels.cu", "linalg.cu"]
CXX_SOURCES = ["engine.cpp", "api.cpp", "serve.cpp", "powmod.cpp"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ({r.returncode})")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "nbgpu.h"))
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _stale(o, [s] + headers) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            _run([NVCC] + NVCC_FLAGS + extra + ["-c", s, "-o", o])
        objs.append(o)
    cxx = shutil.which("g++") or "g++"
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _stale(o, [s] + headers):
            _run([cxx] + CXX_FLAGS + ["-c", s, "-o", o])
        objs.append(o)
    out = os.path.join(LIB, "libnbgpu.so")
    if _stale(out, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", out] + objs + ["-cudart", "static", "-lpthread", "-ldl", "-lrt"])
    # open-loop request generator of the serving benchmark (links libnbgpu.so)
    ls = os.path.join(CSRC, "loadgen.cpp")
    lo = os.path.join(LIB, "libnbgpu_loadgen.so")
    if _stale(lo, [ls, out]):
        _run([cxx] + CXX_FLAGS + ["-shared", ls, "-o", lo, f"-L{LIB}", "-lnbgpu", "-Wl,-rpath,$ORIGIN"])
    # FP64 issue-rate probe used by bench.py for the roofline denominator
    ps = os.path.join(CSRC, "peak.cu")
    po = os.path.join(LIB, "libnbgpu_peak.so")
    if _stale(po, [ps]):
        _run([NVCC] + NVCC_FLAGS + ["-shared", ps, "-o", po, "-cudart", "static"])
    if verbose:
        print(out)
    return out


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
