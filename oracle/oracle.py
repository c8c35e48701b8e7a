"""ctypes wrapper of the FP64 oracle (TEST INFRASTRUCTURE -- never the product).

Loads oracle/liboracle.so and drives it from a compiled-model dump
(mjb200_model_dump, parsed by mjb200.parse_dump).  Parity status: unpinned
(see mjoracle.h).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

_MODEL_INT = ["nq", "nv", "nu", "nbody", "njnt", "ngeom", "nmesh", "npair", "iterations", "ls_iterations", "cone", "integrator", "disableflags"]
_MODEL_PTR = [
    ("body_parentid", "i"), ("body_rootid", "i"), ("body_weldid", "i"), ("body_jntnum", "i"), ("body_jntadr", "i"), ("body_dofnum", "i"),
    ("body_dofadr", "i"), ("body_subtreesize", "i"),
    ("body_pos", "f"), ("body_quat", "f"), ("body_ipos", "f"), ("body_iquat", "f"), ("body_mass", "f"), ("body_inertia", "f"), ("body_invweight0", "f"),
    ("jnt_type", "i"), ("jnt_qposadr", "i"), ("jnt_dofadr", "i"), ("jnt_bodyid", "i"), ("jnt_limited", "i"),
    ("jnt_pos", "f"), ("jnt_axis", "f"), ("jnt_range", "f"), ("jnt_margin", "f"), ("jnt_solref", "f"), ("jnt_solimp", "f"), ("jnt_stiffness", "f"),
    ("dof_bodyid", "i"), ("dof_jntid", "i"), ("dof_parentid", "i"),
    ("dof_armature", "f"), ("dof_damping", "f"), ("dof_frictionloss", "f"), ("dof_invweight0", "f"), ("dof_solref", "f"), ("dof_solimp", "f"),
    ("qpos0", "f"), ("qpos_spring", "f"),
    ("geom_type", "i"), ("geom_bodyid", "i"), ("geom_dataid", "i"),
    ("geom_pos", "f"), ("geom_quat", "f"), ("geom_size", "f"), ("geom_rbound", "f"),
    ("mesh_vertadr", "i"), ("mesh_vertnum", "i"), ("mesh_vert", "f"),
    ("actuator_trnid", "i"), ("actuator_gaintype", "i"), ("actuator_biastype", "i"), ("actuator_ctrllimited", "i"), ("actuator_forcelimited", "i"),
    ("actuator_gear", "f"), ("actuator_gainprm", "f"), ("actuator_biasprm", "f"), ("actuator_ctrlrange", "f"), ("actuator_forcerange", "f"),
    ("pair_int", "i"), ("pair_real", "f"),
]


_EQ_PTR = [("eq_type", "i"), ("eq_obj1", "i"), ("eq_obj2", "i"), ("eq_active", "i"),
           ("eq_data", "f"), ("eq_solref", "f"), ("eq_solimp", "f"), ("eq_invweight", "f")]


_TEN_PTR = [("tendon_adr", "i"), ("tendon_num", "i"), ("tendon_limited", "i"), ("wrap_objid", "i"), ("actuator_trntype", "i"),
            ("wrap_prm", "f"), ("tendon_range", "f"), ("tendon_margin", "f"), ("tendon_frictionloss", "f"), ("tendon_stiffness", "f"),
            ("tendon_damping", "f"), ("tendon_lengthspring", "f"), ("tendon_solref_lim", "f"), ("tendon_solimp_lim", "f"),
            ("tendon_solref_fri", "f"), ("tendon_solimp_fri", "f"), ("tendon_length0", "f"), ("tendon_invweight0", "f")]


_SENS_PTR = [("site_bodyid", "i"), ("sensor_type", "i"), ("sensor_objtype", "i"), ("sensor_objid", "i"), ("sensor_dim", "i"),
             ("sensor_adr", "i"), ("sensor_supported", "i"), ("site_pos", "f"), ("site_quat", "f"), ("magnetic", "f"),
             ("body_gravcomp", "f"), ("wrap_type", "i")]


class OModel(C.Structure):
    _fields_ = ([(n, C.c_int) for n in _MODEL_INT] +
                [("timestep", C.c_double), ("gravity", C.c_double * 3), ("tolerance", C.c_double), ("ls_tolerance", C.c_double),
                 ("impratio", C.c_double), ("meaninertia", C.c_double)] +
                [(n, _ip if k == "i" else _dp) for n, k in _MODEL_PTR] +
                [("neq", C.c_int)] + [(n, _ip if k == "i" else _dp) for n, k in _EQ_PTR] +
                [("ntendon", C.c_int)] + [(n, _ip if k == "i" else _dp) for n, k in _TEN_PTR] +
                [("nsite", C.c_int), ("nsensor", C.c_int)] + [(n, _ip if k == "i" else _dp) for n, k in _SENS_PTR])


class ORand(C.Structure):
    _fields_ = [("mass_scale", _dp), ("friction_scale", C.c_double), ("gain_scale", _dp), ("com_delta", _dp), ("drag_k", _dp)]


_DATA_D = ["qpos", "qvel", "ctrl", "qacc_warmstart", "qacc_predicted",
           "xpos", "xquat", "xmat", "xipos", "ximat", "xanchor", "xaxis", "geom_xpos", "geom_xmat",
           "subtree_com", "cinert", "cdof", "cvel", "cdof_dot", "cacc", "cfrc",
           "M", "qLD", "qfrc_bias", "qfrc_passive", "qfrc_actuator", "qfrc_smooth", "qacc_smooth",
           "contact", "efc_J", "efc_aref", "efc_D", "efc_R", "efc_floss", "efc_force", "efc_jar"]


class OData(C.Structure):
    _fields_ = ([("ncon_max", C.c_int), ("nefc_max", C.c_int)] + [(n, _dp) for n in _DATA_D] + [("efc_type", _ip)] +
                [(n, _dp) for n in ("qacc", "qfrc_constraint", "cfrc_ext", "work")] +
                [(n, C.c_int) for n in ("ncon", "nefc", "niter", "status", "warm_choice", "ncon_dropped", "nefc_dropped")] +
                [("cost_initial", C.c_double), ("cost_final", C.c_double)])


CONTACT_STRIDE = 20


def _load():
    import importlib.util
    spec = importlib.util.spec_from_file_location("mjb_oracle_build", os.path.join(HERE, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    path = mod.build()
    lib = C.CDLL(path)
    for fn in ("oracle_kinematics", "oracle_collide"):
        getattr(lib, fn).argtypes = [C.POINTER(OModel), C.POINTER(OData)]
    for fn in ("oracle_com", "oracle_crb", "oracle_rne", "oracle_smooth_forces", "oracle_make_constraints"):
        getattr(lib, fn).argtypes = [C.POINTER(OModel), C.POINTER(OData), C.POINTER(ORand)]
    lib.oracle_solve.argtypes = [C.POINTER(OModel), C.POINTER(OData), C.c_int]
    lib.oracle_integrate.argtypes = [C.POINTER(OModel), C.POINTER(OData)]
    lib.oracle_step.argtypes = [C.POINTER(OModel), C.POINTER(OData), C.POINTER(ORand), C.c_int]
    lib.oracle_ray.restype = C.c_double
    lib.oracle_ray.argtypes = [C.POINTER(OModel), C.POINTER(OData), _dp, _dp, _ip, _ip]
    lib.oracle_tendon.argtypes = [C.POINTER(OModel), C.POINTER(OData), C.c_int, _dp, _dp, _dp]
    lib.oracle_sensors.argtypes = [C.POINTER(OModel), C.POINTER(OData), _dp, _dp, _dp, _dp, _dp]
    lib.oracle_step_batch.argtypes = [C.POINTER(OModel), C.POINTER(C.POINTER(OData)), C.c_int, C.c_int, C.c_int, C.c_int]
    return lib


lib = _load()


def _ptr(a, kind):
    return a.ctypes.data_as(_ip if kind == "i" else _dp)


def parse_dump(text: str) -> dict:
    """Arrays of a compiled-model dump (the text of mjb200_model_dump: per
    line name, kind i / f, count, values)."""
    out = {}
    for line in text.splitlines():
        parts = line.split()
        if not parts:
            continue
        name, kind, n = parts[0], parts[1], int(parts[2])
        vals = parts[3:3 + n]
        out[name] = np.array([int(v) for v in vals], np.int64) if kind == "i" else np.array([float(v) for v in vals], np.float64)
    return out


def load_dump(name: str) -> dict:
    """A committed model dump from oracle/models/ (see make_model_dumps.py)."""
    with open(os.path.join(HERE, "models", name)) as f:
        return parse_dump(f.read())


class OracleModel:
    """OModel built from a model dump (dict of numpy arrays)."""

    def __init__(self, dump: dict):
        self.dump = dump
        s = dump["sizes"]
        self.nq, self.nv, self.nu, self.nbody, self.njnt, self.ngeom, self.nmesh, self.npair = [int(x) for x in s[:8]]
        self.keep = {}
        m = OModel()
        for n, v in zip(["nq", "nv", "nu", "nbody", "njnt", "ngeom", "nmesh", "npair"], s[:8]):
            setattr(m, n, int(v))
        oi = dump["opt_int"]
        m.iterations, m.ls_iterations, m.cone, m.integrator, m.disableflags = [int(x) for x in oi]
        orr = dump["opt_real"]
        m.timestep = orr[0]
        m.gravity[0], m.gravity[1], m.gravity[2] = orr[1:4]
        m.tolerance, m.ls_tolerance, m.impratio, m.meaninertia = orr[4:8]
        m.neq = int(len(dump.get("eq_type", [])))
        m.ntendon = int(len(dump.get("tendon_adr", [])))
        m.nsite = int(len(dump.get("site_bodyid", [])))
        m.nsensor = int(len(dump.get("sensor_type", [])))
        self.nsensordata = int(np.sum(dump.get("sensor_dim", [])))
        for n, k in _MODEL_PTR + _EQ_PTR + _TEN_PTR + _SENS_PTR:
            a = dump[n] if n in dump else np.zeros(0)
            a = np.ascontiguousarray(a, dtype=np.int32 if k == "i" else np.float64)
            if a.size == 0:
                a = np.zeros(1, a.dtype)
            self.keep[n] = a
            setattr(m, n, _ptr(a, k))
        self.c = m

    def set_option(self, **kw):
        for k, v in kw.items():
            setattr(self.c, k, v)


class OracleEnv:
    """One env's OData with numpy-backed buffers."""

    def __init__(self, om: OracleModel, ncon_max: int = 64, nefc_max: int = 256):
        self.om = om
        nq, nv, nu, nb, nj, ng = om.nq, om.nv, om.nu, om.nbody, om.njnt, om.ngeom
        sizes = dict(qpos=nq, qvel=nv, ctrl=max(nu, 1), qacc_warmstart=nv, xpos=3 * nb, xquat=4 * nb, xmat=9 * nb, xipos=3 * nb, ximat=9 * nb,
                     xanchor=3 * max(nj, 1), xaxis=3 * max(nj, 1), geom_xpos=3 * max(ng, 1), geom_xmat=9 * max(ng, 1), subtree_com=3 * nb,
                     cinert=10 * nb, cdof=6 * max(nv, 1), cvel=6 * nb, cdof_dot=6 * max(nv, 1), cacc=6 * nb, cfrc=6 * nb, M=nv * nv, qLD=nv * nv,
                     qfrc_bias=nv, qfrc_passive=nv, qfrc_actuator=nv, qfrc_smooth=nv, qacc_smooth=nv, contact=CONTACT_STRIDE * ncon_max,
                     efc_J=nefc_max * nv, efc_aref=nefc_max, efc_D=nefc_max, efc_R=nefc_max, efc_floss=nefc_max, efc_force=nefc_max,
                     efc_jar=nefc_max, qacc=nv, qfrc_constraint=nv, cfrc_ext=6 * nb,
                     work=6 * nv * nv + 16 * nv + 8 * nefc_max + 16 * nb + 64)
        self.a = {k: np.zeros(v, np.float64) for k, v in sizes.items()}
        self.a["efc_type"] = np.zeros(nefc_max, np.int32)
        self.a["qpos"][:] = om.dump["qpos0"]
        d = OData()
        d.ncon_max, d.nefc_max = ncon_max, nefc_max
        for k, v in self.a.items():
            setattr(d, k, _ptr(v, "i" if k == "efc_type" else "f"))
        d.qacc_predicted = None
        self.d = d
        self._pred = None

    def ray(self, pnt, vec, include):
        """Nearest hit (t, geom id) at the poses of the last kinematics pass."""
        p = np.ascontiguousarray(pnt, np.float64)
        v = np.ascontiguousarray(vec, np.float64)
        inc = np.ascontiguousarray(include, np.int32)
        g = C.c_int(-1)
        t = lib.oracle_ray(C.byref(self.om.c), C.byref(self.d), _ptr(p, "f"), _ptr(v, "f"), _ptr(inc, "i"), C.byref(g))
        return t, g.value

    def kinematics(self):
        lib.oracle_kinematics(C.byref(self.om.c), C.byref(self.d))

    def tendon(self, t: int):
        """(length, velocity, J[nv]) of tendon t at the current qpos / qvel
        (runs kinematics and the COM pass first)."""
        lib.oracle_kinematics(C.byref(self.om.c), C.byref(self.d))
        lib.oracle_com(C.byref(self.om.c), C.byref(self.d), None)
        ln, vl = C.c_double(), C.c_double()
        J = np.zeros(max(self.om.nv, 1))
        lib.oracle_tendon(C.byref(self.om.c), C.byref(self.d), t, C.byref(ln), C.byref(vl), _ptr(J, "f"))
        return ln.value, vl.value, J[: self.om.nv]

    def step_sensors(self, max_iter: int = 0, rand: ORand | None = None):
        """One step, then the sensordata of its start state; accelerometers
        difference against the previous call's frame velocities (none after
        construction or reset_sensor_history)."""
        q0 = self.a["qpos"].copy()
        v0 = self.a["qvel"].copy()
        self.step(max_iter, rand)
        ns = max(self.om.c.nsensor, 1)
        out = np.zeros(max(self.om.nsensordata, 1))
        lin = np.zeros(3 * ns)
        prev = getattr(self, "_linvel", None)
        lib.oracle_sensors(C.byref(self.om.c), C.byref(self.d), _ptr(q0, "f"), _ptr(v0, "f"), None if prev is None else _ptr(prev, "f"),
                           _ptr(lin, "f"), _ptr(out, "f"))
        self._linvel = lin
        return out[: self.om.nsensordata]

    def reset_sensor_history(self):
        self._linvel = None

    def set_predicted(self, qacc):
        if qacc is None:
            self.d.qacc_predicted = None
            self._pred = None
        else:
            self._pred = np.ascontiguousarray(qacc, np.float64)
            self.d.qacc_predicted = _ptr(self._pred, "f")

    def step(self, max_iter: int = 0, rand: ORand | None = None):
        lib.oracle_step(C.byref(self.om.c), C.byref(self.d), C.byref(rand) if rand else None, max_iter)

    # convenience views
    def contacts(self):
        return self.a["contact"][: CONTACT_STRIDE * self.d.ncon].reshape(-1, CONTACT_STRIDE).copy()

    def efc(self):
        n, nv = self.d.nefc, self.om.nv
        return dict(J=self.a["efc_J"][: n * nv].reshape(n, nv).copy(), aref=self.a["efc_aref"][:n].copy(), D=self.a["efc_D"][:n].copy(),
                    force=self.a["efc_force"][:n].copy(), type=self.a["efc_type"][:n].copy())


class OracleBatch:
    """B envs stepped on host threads (the reference's CPU-pool scheme)."""

    def __init__(self, om: OracleModel, B: int, ncon_max: int = 64, nefc_max: int = 256):
        self.om, self.B = om, B
        self.envs = [OracleEnv(om, ncon_max, nefc_max) for _ in range(B)]
        self.ptrs = (C.POINTER(OData) * B)(*[C.pointer(e.d) for e in self.envs])

    def set_state(self, qpos, qvel):
        for e, env in enumerate(self.envs):
            env.a["qpos"][:] = qpos[e]
            env.a["qvel"][:] = qvel[e]

    def set_ctrl(self, ctrl):
        for e, env in enumerate(self.envs):
            env.a["ctrl"][: self.om.nu] = ctrl[e]

    def state(self):
        return (np.stack([env.a["qpos"].copy() for env in self.envs]), np.stack([env.a["qvel"].copy() for env in self.envs]))

    def step(self, nsub: int = 1, max_iter: int = 0, nthread: int = 1):
        lib.oracle_step_batch(C.byref(self.om.c), self.ptrs, self.B, nsub, max_iter, nthread)
