"""Builds the FP64 oracle (test infrastructure) into oracle/liboracle.so.

    python oracle/build.py

The reference itself cannot be built here (its GPU path needs Vulkan and the
empty extern/mlx_vulkan submodule; its CPU path needs MuJoCo C 3.5.0, which
is not installed), so there is no oracle/_ref build.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRCS = ["o_dyn.c", "o_collide.c", "o_solver.c", "o_ray.c", "o_sensor.c"]
OUT = os.path.join(HERE, "liboracle.so")


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, s) for s in SRCS]
    deps = srcs + [os.path.join(HERE, h) for h in ("mjoracle.h", "o_util.h")]
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(p) for p in deps):
        return OUT
    cmd = ["gcc", "-O2", "-std=c11", "-Wall", "-Wextra", "-fPIC", "-shared", *srcs, "-o", OUT, "-lm", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
