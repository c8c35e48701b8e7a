"""Builds libmjb200.so (host C++ + sm_100a CUDA kernels) in-tree.

    python mujoco-mlx-cpp_b200/build.py [--force]

Host sources compile with g++ -std=c++20, CUDA sources with
nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo; the shared library
links the CUDA runtime statically so it loads without a GPU present (CUDA
calls then report errors).  Objects go to mujoco-mlx-cpp_b200/_build/.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmjb200.so")
BUILD = os.path.join(HERE, "_build")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

CXXFLAGS = ["-std=c++20", "-O2", "-fPIC", "-Wall", "-Wextra", "-fvisibility=hidden", f"-I{CUDA_HOME}/include"]
NVCCFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
             "-gencode", "arch=compute_100a,code=sm_100a", "--expt-relaxed-constexpr"]


def _sources():
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    return cpp, cu


def _headers_mtime():
    t = 0.0
    for d in (CSRC, os.path.join(HERE, "..", "include", "mjmlx")):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh")):
                t = max(t, os.path.getmtime(os.path.join(d, f)))
    return t


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cpp, cu = _sources()
    hdr = _headers_mtime()
    jobs, objs = [], []
    for f in cpp + cu:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr):
            continue
        if f.endswith(".cpp"):
            jobs.append(["g++", *CXXFLAGS, "-c", src, "-o", obj])
        else:
            jobs.append([NVCC, *NVCCFLAGS, "-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for out in ex.map(_compile, jobs):
            if verbose and out:
                print(out, file=sys.stderr)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or jobs or not os.path.exists(OUT) or os.path.getmtime(OUT) < newest:
        _compile([NVCC, "-shared", "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a",
                  "-o", OUT, *objs, "-lpthread", "-ldl", "-lrt"])
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
