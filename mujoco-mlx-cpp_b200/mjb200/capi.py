"""ctypes bindings of libmjb200.so (the C ABI in include/mjmlx/*.h)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libmjb200.so")

_f32p = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int)


class MjmlxModelInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nq", "nv", "nu", "na", "nbody", "njnt", "ngeom", "nsite", "ncon")]


class MjmlxModelOptions(C.Structure):
    _fields_ = [("self_collision", C.c_int), ("max_condim", C.c_int)]


class MjmlxBatchedConfig(C.Structure):
    _fields_ = [("num_envs", C.c_int), ("integrator", C.c_int), ("use_gpu", C.c_int),
                ("solver_iterations", C.c_int), ("domain_rand", C.c_int)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run mujoco-mlx-cpp_b200/build.py (no fallback exists)")
    lib = C.CDLL(LIB_PATH)
    sig = {
        "mjmlx_version": (C.c_char_p, []),
        "mjb200_last_error": (C.c_char_p, []),
        "mjmlx_load_model_from_string": (C.c_void_p, [C.c_char_p]),
        "mjmlx_load_model_from_string_ex": (C.c_void_p, [C.c_char_p, C.POINTER(MjmlxModelOptions)]),
        "mjmlx_load_model": (C.c_void_p, [C.c_char_p]),
        "mjmlx_free_model": (None, [C.c_void_p]),
        "mjmlx_model_info": (MjmlxModelInfo, [C.c_void_p]),
        "mjmlx_model_opt_timestep": (C.c_float, [C.c_void_p]),
        "mjmlx_name2id": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p]),
        "mjb200_model_dump": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    return lib.mjb200_last_error().decode()


def parse_dump(text: str) -> dict:
    out = {}
    for line in text.splitlines():
        parts = line.split()
        if not parts:
            continue
        name, kind, n = parts[0], parts[1], int(parts[2])
        vals = parts[3:3 + n]
        out[name] = np.array([int(v) for v in vals], np.int64) if kind == "i" else np.array([float(v) for v in vals], np.float64)
    return out


class Model:
    def __init__(self, handle):
        if not handle:
            raise RuntimeError("model load failed: " + last_error())
        self.handle = C.c_void_p(handle)
        self.info = lib.mjmlx_model_info(self.handle)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            lib.mjmlx_free_model(h)
            self.handle = None

    @property
    def nq(self):
        return self.info.nq

    @property
    def nv(self):
        return self.info.nv

    @property
    def nu(self):
        return self.info.nu

    def dump(self) -> dict:
        n = lib.mjb200_model_dump(self.handle, None, 0)
        buf = C.create_string_buffer(n)
        lib.mjb200_model_dump(self.handle, buf, n)
        return parse_dump(buf.value.decode())

    def name2id(self, objtype: int, name: str) -> int:
        return lib.mjmlx_name2id(self.handle, objtype, name.encode())


def load_model_from_string(xml: str, self_collision: int = 1, max_condim: int = 0) -> Model:
    opt = MjmlxModelOptions(self_collision, max_condim)
    return Model(lib.mjmlx_load_model_from_string_ex(xml.encode(), C.byref(opt)))


def load_model(path: str) -> Model:
    return Model(lib.mjmlx_load_model(path.encode()))


class BatchedSim:  # filled in by engine bindings below
    pass
