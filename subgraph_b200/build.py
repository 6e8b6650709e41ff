"""Builds the native library (libsubgraph_b200.so) and the sc-main CLI in-tree.

CUDA sources are compiled for sm_100a only; host C++ with the system g++.
Objects go to subgraph_b200/_build/ (git-ignored); the shared library and the
CLI binary land next to this file so they travel with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsubgraph_b200.so")
CLI = os.path.join(HERE, "bin", "sc-main")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH
CXX_FLAGS = ["-std=c++17", "-O3", "-fPIC", "-Wall", "-Wno-unused-function"]

HOST_SOURCES = ["host/graph_io.cpp", "host/plan.cpp", "capi.cpp"]
CUDA_SOURCES = ["engine/kernels.cu", "engine/blocked.cu", "engine/blocked_a.cu", "engine/blocked_b.cu",
                "engine/blocked_c.cu", "engine/blocked_d.cu", "engine/blocked_e.cu", "engine/engine.cu", "engine/batch.cu", "engine/noalloc.cu",
                "engine/input_gpu.cu"]


def _cuda_home() -> str:
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc)))


def _cxx() -> str:
    for c in ("/usr/bin/g++", shutil.which("g++") or ""):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("g++ not found")


def _deps() -> list[str]:
    out = []
    for d, _, files in os.walk(CSRC):
        out += [os.path.join(d, f) for f in files if f.endswith((".hpp", ".cuh", ".h"))]
    out.append(os.path.join(ROOT, "include", "sg_api.h"))
    return out


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    cuda = _cuda_home()
    inc = ["-I" + os.path.join(cuda, "include"), "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    deps = _deps()
    jobs = []
    objs = []
    for src in HOST_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace("/", "_") + ".o")
        objs.append(o)
        if force or _stale(o, [s] + deps):
            jobs.append([_cxx()] + CXX_FLAGS + inc + ["-c", s, "-o", o])
    for src in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace("/", "_") + ".o")
        objs.append(o)
        if force or _stale(o, [s] + deps):
            jobs.append(["nvcc"] + NVCC_FLAGS + inc + ["-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, j) for j in jobs]:
            f.result()
    if force or jobs or _stale(LIB, objs):
        _run(["nvcc", "-shared"] + ARCH + ["-o", LIB] + objs + ["-cudart", "static"])
    cli_src = os.path.join(CSRC, "sc_main.cpp")
    shim = [os.path.join(ROOT, "include", "subgraph_b200", f) for f in sorted(os.listdir(os.path.join(ROOT, "include", "subgraph_b200")))]
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB] + deps + shim)):
        _run([_cxx()] + CXX_FLAGS + ["-I" + os.path.join(ROOT, "include"), cli_src, "-o", CLI,
                                     "-L" + HERE, "-lsubgraph_b200", "-Wl,-rpath,$ORIGIN/.."])
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
