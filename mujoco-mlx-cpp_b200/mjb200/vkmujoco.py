"""The reference's numpy-facing RL module (``vkmujoco``, built from
python/rl_bindings.cpp) over this engine.

RL code written against that module runs on the B200 engine by changing its
import to ``import mjb200.vkmujoco as vkmujoco``.  The functions, classes,
methods, argument names and defaults, array shapes and dtypes are the
reference's (rl_bindings.cpp:233-330), and so are the conditions under which
a call raises RuntimeError: a control array that is not (num_envs, nu), a
reset mask that is not (num_envs,), a state of the wrong shape, per-env
parameters of the wrong shapes or on a sim created without domain_rand,
drag coefficients that are not (n, num_free_joints), rays that are neither
(num_envs, nray, 3) nor (nray, 3), a pack read before set_pack_spec.

Differences, each raising rather than returning something else: the CPU
backend (use_gpu=False) is MuJoCo C in the reference and is not part of this
engine, and camera rendering is graphics, which this engine does not have
(create_camera raises).  frame_skip is accepted and ignored, as in the
reference (frame skipping is step(ctrl, n)).
"""
from __future__ import annotations

import numpy as np

from . import capi

__all__ = ["Model", "BatchedSim", "load_model", "create_batched", "create_camera", "version", "__version__"]


def version() -> str:
    v = capi.lib.mjmlx_version()
    return v.decode() if v else ""


__version__ = version()


class Model:
    """A compiled model (rl_bindings.cpp:233-243): nq, nv, nu, nbody,
    nsensordata, sensors(), name2id(obj_type, name), body_mass(body_id)."""

    def __init__(self, model: capi.Model):
        self._model = model

    @property
    def nq(self) -> int:
        return self._model.info.nq

    @property
    def nv(self) -> int:
        return self._model.info.nv

    @property
    def nu(self) -> int:
        return self._model.info.nu

    @property
    def nbody(self) -> int:
        return self._model.info.nbody

    @property
    def nsensordata(self) -> int:
        return self._model.nsensordata

    def sensors(self):
        """[(name, mjtSensor type, adr, dim), ...]"""
        return self._model.sensors()

    def name2id(self, obj_type: int, name: str) -> int:
        return self._model.name2id(obj_type, name)

    def body_mass(self, body_id: int) -> float:
        return float(capi.lib.mjmlx_model_body_mass(self._model.handle, body_id))


def load_model(xml_path: str, self_collision: bool = True, max_condim: int = 0) -> Model:
    try:
        return Model(capi.load_model(xml_path, 1 if self_collision else 0, max_condim))
    except RuntimeError as e:
        raise RuntimeError(f"vkmujoco: failed to load model {xml_path}: {e}") from None


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class BatchedSim:
    """num_envs copies of one model stepped together (rl_bindings.cpp:49-225)."""

    def __init__(self, sim, model: Model, num_envs: int):
        self._sim = sim
        self._model = model
        self.num_envs = num_envs
        self.nq, self.nv, self.nu, self.nbody = model.nq, model.nv, model.nu, model.nbody
        self._pack_stride = 0

    # ---- stepping and state
    def step(self, ctrl, n: int = 1) -> None:
        if self.nu > 0:
            c = np.asarray(ctrl)
            if c.ndim != 2 or c.shape != (self.num_envs, self.nu):
                raise RuntimeError("vkmujoco: ctrl must have shape (num_envs, nu)")
            self._sim.step(_f32(c), n)
        else:
            self._sim.step(None, n)

    def reset(self, mask) -> None:
        m = np.asarray(mask)
        if m.ndim != 1 or m.shape[0] != self.num_envs:
            raise RuntimeError("vkmujoco: mask must have shape (num_envs,)")
        self._sim.reset(np.ascontiguousarray(m, dtype=np.int32))

    def set_env_qpos(self, env_idx: int, qpos) -> None:
        self._sim.set_env_state(env_idx, qpos=_f32(qpos))

    def set_env_qvel(self, env_idx: int, qvel) -> None:
        self._sim.set_env_state(env_idx, qvel=_f32(qvel))

    def set_state(self, qpos, qvel) -> None:
        q, v = np.asarray(qpos), np.asarray(qvel)
        if q.ndim != 2 or q.shape != (self.num_envs, self.nq):
            raise RuntimeError("vkmujoco: qpos must have shape (num_envs, nq)")
        if v.ndim != 2 or v.shape != (self.num_envs, self.nv):
            raise RuntimeError("vkmujoco: qvel must have shape (num_envs, nv)")
        self._sim.set_state(_f32(q), _f32(v))

    def sync(self) -> None:
        """Wait until the queued steps have finished on the GPU."""
        self._sim.sync()

    def state(self):
        q, v = self._sim.state()
        return q.reshape(self.num_envs, self.nq), v.reshape(self.num_envs, self.nv)

    def _rows(self, name):
        a = self._sim.get(name)
        return a.reshape(self.num_envs, -1)

    def qpos(self):
        return self._rows("qpos")

    def qvel(self):
        return self._rows("qvel")

    def xpos(self):
        return self._rows("xpos")

    def cfrc_ext(self):
        return self._rows("cfrc_ext")

    def qfrc_actuator(self):
        return self._rows("qfrc_actuator")

    def sensordata(self):
        """(num_envs, nsensordata) in MuJoCo's sensor_adr order; (num_envs, 0)
        without sensors."""
        if self._model.nsensordata == 0:
            return np.zeros((self.num_envs, 0), np.float32)
        return self._sim.sensordata()

    # ---- per-env physics parameters
    def set_env_params(self, env_idx=None, mass_scale=None, com_delta=None, friction_scale=None, gain_scale=None) -> None:
        n = self.num_envs if env_idx is None else np.asarray(env_idx).shape[0]

        def check(a, shape, what):
            if a is None:
                return None
            a = np.asarray(a)
            if a.shape != shape:
                raise RuntimeError(f"vkmujoco: {what} must have shape {shape}")
            return a

        ms = check(mass_scale, (n, self.nbody), "mass_scale")
        cd = check(com_delta, (n, self.nbody, 3), "com_delta")
        fs = check(friction_scale, (n,), "friction_scale")
        gs = check(gain_scale, (n, self.nu), "gain_scale")
        idx = None if env_idx is None else np.ascontiguousarray(env_idx, dtype=np.int32)
        if self._sim.set_env_params(idx, mass_scale=ms, friction_scale=fs, gain_scale=gs, com_delta=cd) != 0:
            raise RuntimeError("vkmujoco: set_env_params failed (the sim needs create_batched(domain_rand=True); env_idx must be in range)")

    def num_free_joints(self) -> int:
        return self._sim.num_free_joints()

    def set_free_drag(self, drag_k, env_idx=None) -> None:
        nf = self.num_free_joints()
        n = self.num_envs if env_idx is None else np.asarray(env_idx).shape[0]
        k = np.asarray(drag_k)
        if k.ndim != 2 or k.shape != (n, nf):
            raise RuntimeError("vkmujoco: drag_k must have shape (n, num_free_joints)")
        idx = None if env_idx is None else np.ascontiguousarray(env_idx, dtype=np.int32)
        if self._sim.set_free_drag(_f32(k), idx) != 0:
            raise RuntimeError("vkmujoco: set_free_drag failed (the sim needs create_batched(domain_rand=True) and a free joint)")

    # ---- sensing
    def raycast(self, pnt, vec, bodyexclude: int = -1, geomgroup=None, flg_static: bool = True):
        """Rays (num_envs, nray, 3), or (nray, 3) shared by every env:
        (dist, geomid), each (num_envs, nray)."""
        p, v = np.asarray(pnt), np.asarray(vec)

        def per_env(a, what):
            if a.ndim == 3 and a.shape[0] == self.num_envs and a.shape[2] == 3:
                return a
            if a.ndim == 2 and a.shape[1] == 3:
                return np.broadcast_to(a, (self.num_envs,) + a.shape)
            raise RuntimeError(f"vkmujoco: {what} must have shape (num_envs, nray, 3) or (nray, 3)")

        p, v = per_env(p, "pnt"), per_env(v, "vec")
        if p.shape[1] != v.shape[1]:
            raise RuntimeError("vkmujoco: pnt and vec must have the same number of rays")
        if geomgroup is not None and np.asarray(geomgroup).size != 6:
            raise RuntimeError("vkmujoco: geomgroup must have 6 entries")
        return self._sim.raycast(_f32(p), _f32(v), bodyexclude, geomgroup, 1 if flg_static else 0)

    # ---- packed read-back
    def set_pack_spec(self, body_ids, dof_lo: int, ndof: int) -> int:
        self._pack_stride = self._sim.set_pack_spec(np.ascontiguousarray(body_ids, dtype=np.int32), dof_lo, ndof)
        return self._pack_stride

    def read_pack(self):
        if self._pack_stride <= 0:
            raise RuntimeError("vkmujoco: call set_pack_spec first")
        return self._sim.get_pack()

    def read_pack_into(self, out) -> None:
        """Reads straight into the caller's (num_envs, stride) float32
        array (e.g. a page-locked one)."""
        if self._pack_stride <= 0:
            raise RuntimeError("vkmujoco: call set_pack_spec first")
        if not isinstance(out, np.ndarray) or out.dtype != np.float32 or out.shape != (self.num_envs, self._pack_stride) \
                or not out.flags.c_contiguous:
            raise RuntimeError("vkmujoco: out must be a contiguous float32 array of shape (num_envs, stride)")
        self._sim.get_pack(out)


def create_batched(model: Model, num_envs: int, frame_skip: int = 1, use_gpu: bool = True, solver_iterations: int = 0,
                   domain_rand: bool = False) -> BatchedSim:
    del frame_skip   # frame skipping is step(ctrl, n)
    if not use_gpu:
        raise RuntimeError("vkmujoco: use_gpu=False selects MuJoCo C, which this engine does not include")
    try:
        sim = capi.BatchedSim(model._model, num_envs, solver_iterations=solver_iterations, domain_rand=1 if domain_rand else 0)
    except RuntimeError as e:
        raise RuntimeError(f"vkmujoco: failed to create batched sim: {e}") from None
    return BatchedSim(sim, model, num_envs)


def create_camera(sim: BatchedSim, width: int, height: int):
    raise RuntimeError("vkmujoco: camera rendering is graphics, which this engine does not have")
