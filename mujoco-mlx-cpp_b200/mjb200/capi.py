"""ctypes bindings of libmjb200.so (the C ABI in include/mjmlx/*.h)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MJB200_LIB") or os.path.join(os.path.dirname(_HERE), "libmjb200.so")

_f32p = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int)


class MjmlxModelInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nq", "nv", "nu", "na", "nbody", "njnt", "ngeom", "nsite", "ncon")]


class MjmlxModelOptions(C.Structure):
    _fields_ = [("self_collision", C.c_int), ("max_condim", C.c_int)]


class MjmlxBatchedConfig(C.Structure):
    _fields_ = [("num_envs", C.c_int), ("integrator", C.c_int), ("use_gpu", C.c_int),
                ("solver_iterations", C.c_int), ("domain_rand", C.c_int)]


class MjbEngineConfig(C.Structure):
    _fields_ = [("warps_per_block", C.c_int), ("persistent", C.c_int), ("blocks_per_sm", C.c_int), ("ncon_max", C.c_int),
                ("nefc_max", C.c_int), ("use_graph", C.c_int), ("record", C.c_int), ("warmstart", C.c_int),
                ("tolerance", C.c_double), ("max_iter", C.c_int), ("lockstep", C.c_int), ("predict_every", C.c_int)]


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
        "mjmlx_load_model_ex": (C.c_void_p, [C.c_char_p, C.POINTER(MjmlxModelOptions)]),
        "mjmlx_default_model_options": (MjmlxModelOptions, []),
        "mjmlx_model_body_mass": (C.c_float, [C.c_void_p, C.c_int]),
        "mjmlx_free_model": (None, [C.c_void_p]),
        "mjmlx_model_info": (MjmlxModelInfo, [C.c_void_p]),
        "mjmlx_model_opt_timestep": (C.c_float, [C.c_void_p]),
        "mjmlx_name2id": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p]),
        "mjb200_model_dump": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
        "mjmlx_batched_create": (C.c_void_p, [C.c_void_p, C.POINTER(MjmlxBatchedConfig)]),
        "mjmlx_batched_free": (None, [C.c_void_p]),
        "mjmlx_batched_step": (None, [C.c_void_p, _f32p]),
        "mjmlx_batched_step_n": (None, [C.c_void_p, _f32p, C.c_int]),
        "mjmlx_batched_reset": (None, [C.c_void_p, _i32p]),
        "mjmlx_batched_get_state": (None, [C.c_void_p, _f32p, _f32p, _i32p, _i32p]),
        "mjmlx_batched_set_state": (None, [C.c_void_p, _f32p, _f32p]),
        "mjmlx_batched_set_env_qpos": (None, [C.c_void_p, C.c_int, _f32p, C.c_int]),
        "mjmlx_batched_set_env_qvel": (None, [C.c_void_p, C.c_int, _f32p, C.c_int]),
        "mjmlx_batched_set_env_params": (C.c_int, [C.c_void_p, _i32p, C.c_int, _f32p, _f32p, _f32p, _f32p]),
        "mjmlx_batched_set_free_drag": (C.c_int, [C.c_void_p, _i32p, C.c_int, _f32p]),
        "mjmlx_batched_num_free_joints": (C.c_int, [C.c_void_p]),
        "mjmlx_batched_grad_step": (None, [C.c_void_p, _f32p]),
        "mjmlx_batched_set_pack_spec": (C.c_int, [C.c_void_p, _i32p, C.c_int, C.c_int, C.c_int]),
        "mjmlx_batched_get_pack": (C.c_int, [C.c_void_p, _f32p]),
        "mjmlx_batched_raycast": (C.c_int, [C.c_void_p, _f32p, _f32p, C.c_int, C.c_int, C.POINTER(C.c_ubyte), C.c_int, _f32p, _i32p]),
        "mjmlx_batched_eval_state": (None, [C.c_void_p]),
        "mjb200_default_engine_config": (MjbEngineConfig, []),
        "mjb200_batched_create_multi": (C.c_void_p, [C.POINTER(C.c_void_p), _i32p, C.c_int, C.POINTER(MjmlxBatchedConfig), C.POINTER(MjbEngineConfig)]),
        "mjb200_batched_configure": (C.c_int, [C.c_void_p, C.POINTER(MjbEngineConfig)]),
        "mjb200_batched_get_config": (C.c_int, [C.c_void_p, C.POINTER(MjbEngineConfig)]),
        "mjb200_batched_layout": (C.c_int, [C.c_void_p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p]),
        "mjb200_batched_step_device": (C.c_int, [C.c_void_p, C.c_int]),
        "mjb200_batched_step_device_ctrl": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
        "mjb200_warmstart_create": (C.c_void_p, [C.c_int, C.c_int, C.c_ulonglong]),
        "mjb200_warmstart_free": (None, [C.c_void_p]),
        "mjb200_warmstart_input_width": (C.c_int, [C.c_void_p]),
        "mjb200_warmstart_layout": (C.c_int, [C.c_void_p, _i32p, _i32p, _i32p]),
        "mjb200_warmstart_dims": (C.c_int, [C.c_void_p] + [_i32p] * 6),
        "mjb200_warmstart_get_params": (C.c_int, [C.c_void_p, _f32p]),
        "mjb200_warmstart_set_params": (C.c_int, [C.c_void_p, _f32p]),
        "mjb200_warmstart_set_normalization": (C.c_int, [C.c_void_p, _f32p, _f32p, _f32p, _f32p]),
        "mjb200_warmstart_get_normalization": (C.c_int, [C.c_void_p, _f32p, _f32p, _f32p, _f32p]),
        "mjb200_warmstart_fit_normalization": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
        "mjb200_warmstart_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
        "mjb200_warmstart_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, _f32p, _f32p]),
        "mjb200_warmstart_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_ulonglong, _f32p]),
        "mjb200_batched_warmstart_collect": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int]),
        "mjb200_batched_set_warmstart": (C.c_int, [C.c_void_p, C.c_void_p]),
        "mjb200_batched_get_warmstart_debug": (C.c_int, [C.c_void_p, _f32p, _f32p]),
        "mjb200_warmstart_predict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
        "mjb200_gemm_bf16": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
        "mjb200_gemm_bf16_gated": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_double, C.c_void_p,
                                             C.c_void_p]),
        "mjb200_batched_get_qacc_warmstart": (C.c_int, [C.c_void_p, _f32p]),
        "mjb200_batched_set_qacc_warmstart": (C.c_int, [C.c_void_p, _f32p]),
        "mjb200_batched_pack_device": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
        "mjb200_batched_autotune": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f32p]),
        "mjb200_batched_autotune_cached": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
        "mjb200_batched_step_warmstart": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
        "mjb200_batched_step_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
        "mjb200_batched_device_state": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
        "mjb200_batched_stream": (C.c_void_p, [C.c_void_p]),
        "mjb200_batched_launch_shape": (C.c_int, [C.c_void_p, _i32p, _i32p, _i32p, _i32p]),
        "mjb200_batched_stats": (C.c_int, [C.c_void_p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p]),
        "mjb200_batched_get_qacc": (_f32p, [C.c_void_p, _i32p]),
        "mjb200_batched_set_debug": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
        "mjb200_batched_stage_timing": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_ulonglong)]),
        "mjb200_batched_get_debug": (C.c_int, [C.c_void_p, _f32p, _f32p, _f32p]),
    }
    sig.update({
        "mjmlx_model_nsensor": (C.c_int, [C.c_void_p]),
        "mjmlx_model_nsensordata": (C.c_int, [C.c_void_p]),
        "mjmlx_model_sensor_name": (C.c_char_p, [C.c_void_p, C.c_int]),
        "mjmlx_model_sensor_type": (C.c_int, [C.c_void_p, C.c_int]),
        "mjmlx_model_sensor_adr": (C.c_int, [C.c_void_p, C.c_int]),
        "mjmlx_model_sensor_dim": (C.c_int, [C.c_void_p, C.c_int]),
        "mjmlx_batched_nsensordata": (C.c_int, [C.c_void_p]),
        "mjb200_batched_sensordata_device": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), _i32p]),
    })
    for g in ("qpos", "qvel", "xpos", "xquat", "subtree_com", "cinert", "cvel", "qfrc_actuator", "cfrc_ext", "sensordata"):
        sig[f"mjmlx_batched_get_{g}"] = (_f32p, [C.c_void_p, _i32p])
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

    @property
    def nsensordata(self) -> int:
        return lib.mjmlx_model_nsensordata(self.handle)

    def sensors(self):
        """[(name, mjtSensor type, adr, dim)] of the model's sensors."""
        out = []
        for i in range(lib.mjmlx_model_nsensor(self.handle)):
            nm = lib.mjmlx_model_sensor_name(self.handle, i)
            out.append((nm.decode() if nm else "", lib.mjmlx_model_sensor_type(self.handle, i), lib.mjmlx_model_sensor_adr(self.handle, i),
                        lib.mjmlx_model_sensor_dim(self.handle, i)))
        return out


def load_model_from_string(xml: str, self_collision: int = 1, max_condim: int = 0) -> Model:
    opt = MjmlxModelOptions(self_collision, max_condim)
    return Model(lib.mjmlx_load_model_from_string_ex(xml.encode(), C.byref(opt)))


def load_model(path: str, self_collision: int = 1, max_condim: int = 0) -> Model:
    opt = MjmlxModelOptions(self_collision, max_condim)
    return Model(lib.mjmlx_load_model_ex(path.encode(), C.byref(opt)))


def _fp(a):
    return None if a is None else a.ctypes.data_as(_f32p)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_i32p)


def engine_config(**kw) -> MjbEngineConfig:
    c = lib.mjb200_default_engine_config()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


class WarmStart:
    """Learned Newton warm-start network (mjb200_warmstart.h).  Device arrays
    are passed as integer device pointers (e.g. torch tensor data_ptr())."""

    def __init__(self, in_raw: int, nout: int, seed: int = 0):
        h = lib.mjb200_warmstart_create(in_raw, nout, seed)
        if not h:
            raise RuntimeError(last_error())
        self.handle = C.c_void_p(h)
        d = [C.c_int() for _ in range(6)]
        lib.mjb200_warmstart_dims(self.handle, *[C.byref(x) for x in d])
        self.in_raw, self.in_pad, self.hidden, self.nout, self.out_pad, self.nparams = [x.value for x in d]

    def close(self):
        h = getattr(self, "handle", None)
        if h:
            lib.mjb200_warmstart_free(h)
            self.handle = None

    def __del__(self):
        self.close()

    def _ok(self, rc):
        if rc < 0:
            raise RuntimeError(last_error())
        return rc

    def get_params(self):
        p = np.zeros(self.nparams, np.float32)
        self._ok(lib.mjb200_warmstart_get_params(self.handle, _fp(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparams
        self._ok(lib.mjb200_warmstart_set_params(self.handle, _fp(p)))

    def set_normalization(self, in_mean, in_std, out_mean, out_std):
        a = [np.ascontiguousarray(x, np.float32) for x in (in_mean, in_std, out_mean, out_std)]
        self._ok(lib.mjb200_warmstart_set_normalization(self.handle, *[_fp(x) for x in a]))

    def get_normalization(self):
        a = [np.zeros(self.in_raw, np.float32), np.zeros(self.in_raw, np.float32), np.zeros(self.nout, np.float32), np.zeros(self.nout, np.float32)]
        self._ok(lib.mjb200_warmstart_get_normalization(self.handle, *[_fp(x) for x in a]))
        return a

    def fit_normalization(self, xraw_ptr: int, traw_ptr: int, n: int):
        self._ok(lib.mjb200_warmstart_fit_normalization(self.handle, C.c_void_p(xraw_ptr), C.c_void_p(traw_ptr), n))

    def forward(self, xraw_ptr: int, n: int, y_ptr: int):
        self._ok(lib.mjb200_warmstart_forward(self.handle, C.c_void_p(xraw_ptr), n, C.c_void_p(y_ptr)))

    def gradients(self, xraw_ptr: int, traw_ptr: int, n: int):
        g = np.zeros(self.nparams, np.float32)
        loss = np.zeros(1, np.float32)
        self._ok(lib.mjb200_warmstart_gradients(self.handle, C.c_void_p(xraw_ptr), C.c_void_p(traw_ptr), n, _fp(g), _fp(loss)))
        return float(loss[0]), g

    def predict(self, feat_ptr: int, fstride: int, nfeat: int, ctrl_ptr: int, nu: int, prev_ptr: int, pred_ptr: int, B: int, fused: bool = True):
        self._ok(lib.mjb200_warmstart_predict(self.handle, C.c_void_p(feat_ptr), fstride, nfeat, C.c_void_p(ctrl_ptr), nu, C.c_void_p(prev_ptr),
                                              C.c_void_p(pred_ptr), B, 1 if fused else 0))

    def train(self, xraw_ptr: int, traw_ptr: int, n: int, epochs: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0):
        hist = np.zeros(max(epochs, 1), np.float32)
        steps = self._ok(lib.mjb200_warmstart_train(self.handle, C.c_void_p(xraw_ptr), C.c_void_p(traw_ptr), n, epochs, batch, lr, seed, _fp(hist)))
        return steps, hist


def gemm_bf16(a_ptr: int, b_ptr: int, c_ptr: int, M: int, N: int, K: int, stream: int | None = None) -> int:
    return lib.mjb200_gemm_bf16(C.c_void_p(a_ptr), C.c_void_p(b_ptr), C.c_void_p(c_ptr), M, N, K, C.c_void_p(stream))


class BatchedSim:
    """Batched simulation on the CUDA engine (mirrors the reference's Python
    BatchedSim: step(ctrl, n), state(), set_state())."""

    def __init__(self, models, counts=None, solver_iterations: int = 0, domain_rand: int = 0, integrator: int = 0, **engine_kw):
        if isinstance(models, Model):
            models = [models]
            counts = [counts if counts is not None else 1]
        self.models = list(models)
        self.counts = list(counts)
        cfg = MjmlxBatchedConfig(int(sum(self.counts)), integrator, 1, solver_iterations, domain_rand)
        ecfg = engine_config(**engine_kw)
        arr = (C.c_void_p * len(self.models))(*[m.handle.value for m in self.models])
        cnt = np.ascontiguousarray(self.counts, np.int32)
        h = lib.mjb200_batched_create_multi(arr, _ip(cnt), len(self.models), C.byref(cfg), C.byref(ecfg))
        if not h:
            raise RuntimeError("batched create failed: " + last_error())
        self.handle = C.c_void_p(h)
        n, tq, tv, tu = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        lib.mjb200_batched_layout(self.handle, C.byref(n), C.byref(tq), C.byref(tv), C.byref(tu), None, None, None)
        self.num_envs, self.total_q, self.total_v, self.total_u = n.value, tq.value, tv.value, tu.value
        self.qadr = np.zeros(self.num_envs, np.int32)
        self.vadr = np.zeros(self.num_envs, np.int32)
        self.uadr = np.zeros(self.num_envs, np.int32)
        lib.mjb200_batched_layout(self.handle, None, None, None, None, _ip(self.qadr), _ip(self.vadr), _ip(self.uadr))
        self.uniform = len(self.models) == 1

    def close(self):
        h = getattr(self, "handle", None)
        if h:
            lib.mjmlx_batched_free(h)
            self.handle = None

    def __del__(self):
        self.close()

    # ---- stepping
    def step(self, ctrl=None, n: int = 1):
        c = None if ctrl is None else np.ascontiguousarray(ctrl, np.float32).reshape(-1)
        if c is not None and c.size != self.total_u:
            raise ValueError(f"ctrl must have {self.total_u} values")
        lib.mjmlx_batched_step_n(self.handle, _fp(c), n)

    def step_device(self, n: int = 1):
        if lib.mjb200_batched_step_device(self.handle, n) != 0:
            raise RuntimeError(last_error())

    def step_device_ctrl(self, ctrl_ptr: int, n: int = 1):
        if lib.mjb200_batched_step_device_ctrl(self.handle, C.c_void_p(ctrl_ptr), n) != 0:
            raise RuntimeError(last_error())

    def step_noalloc(self, qpos_ptr: int, qvel_ptr: int, ctrl_ptr: int, warm_ptr: int, n: int = 1, stream: int | None = None) -> int:
        """Allocation-free step on caller-owned device buffers; returns the C
        status (0 ok, -1 bad arguments, -2 too many envs, -3 CUDA error)."""
        return lib.mjb200_batched_step_noalloc(self.handle, C.c_void_p(qpos_ptr), C.c_void_p(qvel_ptr), C.c_void_p(ctrl_ptr),
                                               C.c_void_p(warm_ptr), n, C.c_void_p(stream))

    def qacc_warmstart(self):
        out = np.zeros(self.total_v, np.float32)
        if lib.mjb200_batched_get_qacc_warmstart(self.handle, _fp(out)) != 0:
            raise RuntimeError(last_error())
        return out

    def set_qacc_warmstart(self, qacc):
        a = np.ascontiguousarray(qacc, np.float32).reshape(-1)
        if a.size != self.total_v or lib.mjb200_batched_set_qacc_warmstart(self.handle, _fp(a)) != 0:
            raise RuntimeError("set_qacc_warmstart: " + last_error())

    def autotune(self, nsub: int = 4, reps: int = 3):
        """Times the launch-shape candidates and keeps the fastest; returns
        [(warps_per_block, lockstep, ms per launch)]."""
        w = np.zeros(16, np.int32)
        l = np.zeros(16, np.int32)
        t = np.zeros(16, np.float32)
        n = lib.mjb200_batched_autotune(self.handle, nsub, reps, 16, _ip(w), _ip(l), _fp(t))
        if n < 0:
            raise RuntimeError(last_error())
        return [(int(w[i]), int(l[i]), float(t[i])) for i in range(n)]

    def autotune_cached(self, nsub: int = 4, reps: int = 3) -> bool:
        """The autotuner's choice from the process-wide cache (True) or tuned
        now and stored (False)."""
        r = lib.mjb200_batched_autotune_cached(self.handle, nsub, reps)
        if r < 0:
            raise RuntimeError(last_error())
        return r == 1

    def step_warmstart(self, qacc_ptr: int, n: int = 1):
        if lib.mjb200_batched_step_warmstart(self.handle, C.c_void_p(qacc_ptr), n) != 0:
            raise RuntimeError(last_error())

    # ---- packed read-back
    def set_pack_spec(self, body_ids, dof_lo: int, ndof: int) -> int:
        b = np.ascontiguousarray(body_ids, np.int32)
        stride = lib.mjmlx_batched_set_pack_spec(self.handle, _ip(b), len(b), dof_lo, ndof)
        if stride < 0:
            raise RuntimeError("set_pack_spec: " + last_error())
        self.pack_stride = stride
        return stride

    def get_pack(self, out=None):
        """Packed rows [num_envs, stride]; out: optional contiguous float32
        array of that shape to fill (e.g. a page-locked one)."""
        if out is None:
            out = np.zeros((self.num_envs, self.pack_stride), np.float32)
        elif out.dtype != np.float32 or not out.flags.c_contiguous or out.size != self.num_envs * self.pack_stride:
            raise ValueError("out must be a contiguous float32 array of num_envs x stride values")
        if lib.mjmlx_batched_get_pack(self.handle, _fp(out)) != 0:
            raise RuntimeError("get_pack: " + last_error())
        return out

    def num_free_joints(self) -> int:
        return lib.mjmlx_batched_num_free_joints(self.handle)

    def pack_device(self) -> int:
        """Device pointer of the packed rows (num_envs x stride floats)."""
        p = C.c_void_p()
        if lib.mjb200_batched_pack_device(self.handle, C.byref(p)) != 0:
            raise RuntimeError("pack_device: " + last_error())
        return p.value

    def sensordata_pointer(self):
        """(device pointer, float count) of every env's sensordata."""
        p = C.c_void_p()
        n = C.c_int()
        if lib.mjb200_batched_sensordata_device(self.handle, C.byref(p), C.byref(n)) != 0:
            raise RuntimeError("sensordata_device: " + last_error())
        return p.value, n.value

    def raycast(self, pnt, vec, bodyexclude: int = -1, geomgroup=None, flg_static: int = 1):
        """Rays pnt/vec [num_envs, nray, 3] (world frame, per env) against each
        env's geoms at its current qpos: (dist [num_envs, nray], geom id)."""
        p = np.ascontiguousarray(pnt, np.float32)
        v = np.ascontiguousarray(vec, np.float32)
        nray = p.shape[1]
        dist = np.zeros((self.num_envs, nray), np.float32)
        gid = np.zeros((self.num_envs, nray), np.int32)
        gg = None if geomgroup is None else np.ascontiguousarray(geomgroup, np.uint8)
        rc = lib.mjmlx_batched_raycast(self.handle, _fp(p), _fp(v), nray, bodyexclude,
                                       None if gg is None else gg.ctypes.data_as(C.POINTER(C.c_ubyte)), flg_static, _fp(dist), _ip(gid))
        if rc != 0:
            raise RuntimeError("raycast: " + last_error())
        return dist, gid

    # ---- learned warm start
    def warmstart_input_width(self) -> int:
        return lib.mjb200_warmstart_input_width(self.handle)

    def warmstart_layout(self):
        """(in_raw, nout, rows_per_env) of the learned warm start for this sim."""
        d = [C.c_int() for _ in range(3)]
        if lib.mjb200_warmstart_layout(self.handle, *[C.byref(x) for x in d]) < 0:
            raise RuntimeError(last_error())
        return tuple(x.value for x in d)

    def warmstart_collect(self, ctrl_ptr: int, nctrl: int, substeps_per_ctrl: int, xraw_ptr: int, traw_ptr: int, max_rows: int) -> int:
        rc = lib.mjb200_batched_warmstart_collect(self.handle, C.c_void_p(ctrl_ptr), nctrl, substeps_per_ctrl, C.c_void_p(xraw_ptr),
                                                  C.c_void_p(traw_ptr), max_rows)
        if rc < 0:
            raise RuntimeError(last_error())
        return rc

    def set_warmstart(self, net):
        self._warmstart = net
        if lib.mjb200_batched_set_warmstart(self.handle, net.handle if net is not None else None) != 0:
            raise RuntimeError(last_error())

    def warmstart_debug(self):
        """(features [num_envs, in_raw], prediction [total_v]) the fused
        inference used on the last substep (debug capture on)."""
        width = lib.mjb200_warmstart_input_width(self.handle)
        f = np.zeros((self.num_envs, width), np.float32)
        p = np.zeros(self.total_v, np.float32)
        if lib.mjb200_batched_get_warmstart_debug(self.handle, _fp(f), _fp(p)) < 0:
            raise RuntimeError("warmstart_debug: " + last_error())
        return f, p

    def sync(self):
        lib.mjmlx_batched_eval_state(self.handle)

    # ---- state
    def state(self, out=None):
        """(qpos, qvel) of every env.  out: optional preallocated contiguous
        float32 arrays (qpos, qvel) of total_q / total_v values to copy into,
        e.g. page-locked ones for a direct device-to-host DMA."""
        if out is None:
            qpos = np.zeros(self.total_q, np.float32)
            qvel = np.zeros(self.total_v, np.float32)
        else:
            qpos, qvel = out
            if qpos.dtype != np.float32 or qvel.dtype != np.float32 or not (qpos.flags.c_contiguous and qvel.flags.c_contiguous) \
                    or qpos.size != self.total_q or qvel.size != self.total_v:
                raise ValueError("out must be contiguous float32 arrays of total_q and total_v values")
        lib.mjmlx_batched_get_state(self.handle, _fp(qpos), _fp(qvel), None, None)
        if self.uniform:
            return qpos.reshape(self.num_envs, -1), qvel.reshape(self.num_envs, -1)
        return qpos, qvel

    def set_state(self, qpos=None, qvel=None):
        qp = None if qpos is None else np.ascontiguousarray(qpos, np.float32).reshape(-1)
        qv = None if qvel is None else np.ascontiguousarray(qvel, np.float32).reshape(-1)
        lib.mjmlx_batched_set_state(self.handle, _fp(qp), _fp(qv))

    def set_env_state(self, env: int, qpos=None, qvel=None):
        """One env's qpos / qvel (mjmlx_batched_set_env_qpos / _qvel)."""
        if qpos is not None:
            a = np.ascontiguousarray(qpos, np.float32).reshape(-1)
            lib.mjmlx_batched_set_env_qpos(self.handle, env, _fp(a), a.size)
        if qvel is not None:
            a = np.ascontiguousarray(qvel, np.float32).reshape(-1)
            lib.mjmlx_batched_set_env_qvel(self.handle, env, _fp(a), a.size)

    def reset(self, mask):
        m = np.ascontiguousarray(mask, np.int32)
        lib.mjmlx_batched_reset(self.handle, _ip(m))

    def get(self, name: str):
        n = C.c_int()
        if name == "qacc":
            p = lib.mjb200_batched_get_qacc(self.handle, C.byref(n))
        else:
            p = getattr(lib, f"mjmlx_batched_get_{name}")(self.handle, C.byref(n))
        if not p:
            raise RuntimeError(f"get {name} failed: " + last_error())
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    def sensordata(self):
        """Sensor values [num_envs, nsensordata] (uniform batch) of the last
        step's start state."""
        nsd = lib.mjmlx_batched_nsensordata(self.handle)
        if nsd <= 0:
            return np.zeros((self.num_envs, 0), np.float32)
        return self.get("sensordata").reshape(self.num_envs, nsd)

    def stats(self):
        B = self.num_envs
        out = {k: np.zeros(B, np.int32) for k in ("status", "niter_sum", "niter_max", "ncon", "nefc", "warm_choice")}
        lib.mjb200_batched_stats(self.handle, *[_ip(out[k]) for k in ("status", "niter_sum", "niter_max", "ncon", "nefc", "warm_choice")])
        return out

    def set_env_params(self, env_idx=None, mass_scale=None, friction_scale=None, gain_scale=None, com_delta=None):
        n = self.num_envs if env_idx is None else len(env_idx)
        ei = None if env_idx is None else np.ascontiguousarray(env_idx, np.int32)
        conv = lambda a: None if a is None else np.ascontiguousarray(a, np.float32).reshape(-1)
        ms, fs, gs, cd = conv(mass_scale), conv(friction_scale), conv(gain_scale), conv(com_delta)
        return lib.mjmlx_batched_set_env_params(self.handle, _ip(ei), n, _fp(ms), _fp(cd), _fp(fs), _fp(gs))

    def grad_step(self):
        """d(qvel after one step) / d(ctrl) per env, [num_envs, nv, nu]."""
        m = self.models[0]
        out = np.zeros((self.num_envs, m.nv, m.nu), np.float32)
        lib.mjmlx_batched_grad_step(self.handle, _fp(out))
        return out

    def set_free_drag(self, drag_k, env_idx=None):
        """Quadratic drag coefficients [n, nfree] of the free joints."""
        n = self.num_envs if env_idx is None else len(env_idx)
        ei = None if env_idx is None else np.ascontiguousarray(env_idx, np.int32)
        dk = np.ascontiguousarray(drag_k, np.float32).reshape(-1)
        return lib.mjmlx_batched_set_free_drag(self.handle, _ip(ei), n, _fp(dk))

    # ---- debug capture
    def set_debug(self, ncon_max: int = 32, nefc_max: int = 128):
        self.dbg = (ncon_max, nefc_max)
        lib.mjb200_batched_set_debug(self.handle, ncon_max, nefc_max)

    def get_debug(self):
        nc, ne = self.dbg
        B = self.num_envs
        nvmax = max(m.nv for m in self.models)
        con = np.zeros((B, nc, 16), np.float32)
        efc = np.zeros((B, ne, 4), np.float32)
        vec = np.zeros((B, 4, nvmax), np.float32)
        lib.mjb200_batched_get_debug(self.handle, _fp(con), _fp(efc), _fp(vec))
        return con, efc, vec

    def configure(self, **kw):
        c = MjbEngineConfig()
        lib.mjb200_batched_get_config(self.handle, C.byref(c))
        for k, v in kw.items():
            setattr(c, k, v)
        if lib.mjb200_batched_configure(self.handle, C.byref(c)) != 0:
            raise RuntimeError(last_error())

    STAGES = ("finish_kin", "collision", "com_crb", "rne_forces", "qacc_smooth", "constraints", "fused_warmstart", "newton", "x8", "x9", "x10", "x11",
              "x12", "x13", "x14", "x15")

    def stage_timing(self, enable: int = -1):
        out = (C.c_ulonglong * 16)()
        lib.mjb200_batched_stage_timing(self.handle, enable, out)
        return dict(zip(self.STAGES, [int(x) for x in out]))

    def launch_shape(self):
        g, w, s, p = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        lib.mjb200_batched_launch_shape(self.handle, C.byref(g), C.byref(w), C.byref(s), C.byref(p))
        return dict(grid=g.value, warps_per_block=w.value, smem_bytes=s.value, persistent=p.value)

    def device_state(self):
        ptrs = [C.c_void_p() for _ in range(4)]
        lib.mjb200_batched_device_state(self.handle, *[C.byref(p) for p in ptrs])
        return [p.value for p in ptrs]

    def stream(self):
        return lib.mjb200_batched_stream(self.handle)
