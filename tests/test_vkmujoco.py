"""mjb200.vkmujoco, the mirror of the reference's RL module (vkmujoco from
python/rl_bindings.cpp), on the CPU.

Model loading and the model queries run for real (the compiler needs no
GPU).  The sim wrapper's own logic (shape checks, broadcasting, routing and
dtypes) is run over a recording stand-in for mjb200.BatchedSim, whose
methods the GPU tests cover; without a GPU, creating a real sim must fail
cleanly.
"""
import numpy as np
import pytest

import mjb200
from mjb200 import vkmujoco

# the reference binding's public surface (rl_bindings.cpp:233-330)
REF_MODEL = {"nq", "nv", "nu", "nbody", "nsensordata", "sensors", "name2id", "body_mass"}
REF_SIM = {"step", "reset", "set_env_qpos", "set_env_qvel", "set_state", "set_env_params", "set_free_drag", "num_free_joints", "sync",
           "state", "qpos", "qvel", "xpos", "cfrc_ext", "sensordata", "qfrc_actuator", "raycast", "set_pack_spec", "read_pack",
           "read_pack_into"}
REF_MODULE = {"load_model", "create_batched", "create_camera", "version", "__version__", "Model", "BatchedSim"}


def test_public_surface_matches_the_reference():
    assert REF_MODULE <= set(dir(vkmujoco))
    assert REF_MODEL <= set(dir(vkmujoco.Model))
    assert REF_SIM <= set(dir(vkmujoco.BatchedSim))


@pytest.fixture(scope="module")
def quad_file(tmp_path_factory):
    p = tmp_path_factory.mktemp("mjcf") / "quadruped.xml"
    p.write_text(mjb200.models.quadruped_xml())
    return str(p)


def test_load_model_and_queries(quad_file):
    m = vkmujoco.load_model(quad_file)
    assert (m.nq, m.nv, m.nu, m.nbody) == (19, 18, 12, 14)
    d = mjb200.load_model_from_string(mjb200.models.quadruped_xml()).dump()
    for b in range(14):
        assert m.body_mass(b) == pytest.approx(d["body_mass"][b], rel=1e-6)
    assert m.name2id(1, "trunk") == 1 and m.name2id(1, "no_such_body") == -1
    assert m.nsensordata == 0 and m.sensors() == []
    # self_collision off drops the pairs between geoms of one tree
    m0 = vkmujoco.load_model(quad_file, self_collision=False)
    assert (m0.nq, m0.nv) == (19, 18)
    assert int(m0._model.dump()["sizes"][7]) < int(m._model.dump()["sizes"][7]) == 79


def test_load_failures_and_unavailable_paths(tmp_path, quad_file):
    with pytest.raises(RuntimeError):
        vkmujoco.load_model(str(tmp_path / "missing.xml"))
    m = vkmujoco.load_model(quad_file)
    with pytest.raises(RuntimeError):
        vkmujoco.create_batched(m, 4, use_gpu=False)
    import torch

    if not torch.cuda.is_available():
        with pytest.raises(RuntimeError):
            vkmujoco.create_batched(m, 4)       # no GPU: the engine refuses
    with pytest.raises(RuntimeError):
        vkmujoco.create_camera(None, 64, 48)
    assert vkmujoco.version() == vkmujoco.__version__ and vkmujoco.version()


class FakeSim:
    """Records the calls the wrapper makes to mjb200.BatchedSim."""

    def __init__(self, B, nq, nv, nu, nfree=1):
        self.B, self.nq, self.nv, self.nu, self.nfree = B, nq, nv, nu, nfree
        self.calls = []
        self.stride = 0

    def step(self, ctrl, n):
        self.calls.append(("step", None if ctrl is None else (ctrl.dtype, ctrl.shape), n))

    def reset(self, mask):
        self.calls.append(("reset", mask.dtype, mask.shape))

    def set_env_state(self, env, qpos=None, qvel=None):
        self.calls.append(("set_env_state", env, None if qpos is None else qpos.shape, None if qvel is None else qvel.shape))

    def set_state(self, q, v):
        self.calls.append(("set_state", q.dtype, q.shape, v.shape))

    def sync(self):
        self.calls.append(("sync",))

    def state(self):
        return np.zeros((self.B, self.nq), np.float32), np.zeros((self.B, self.nv), np.float32)

    def get(self, name):
        width = {"qpos": self.nq, "qvel": self.nv, "xpos": 3 * 14, "cfrc_ext": 6 * 14, "qfrc_actuator": self.nv}[name]
        return np.arange(self.B * width, dtype=np.float32)

    def sensordata(self):
        return np.zeros((self.B, 0), np.float32)

    def set_env_params(self, idx, mass_scale=None, friction_scale=None, gain_scale=None, com_delta=None):
        self.calls.append(("set_env_params", None if idx is None else idx.dtype, mass_scale is not None, com_delta is not None))
        return 0

    def num_free_joints(self):
        return self.nfree

    def set_free_drag(self, k, idx):
        self.calls.append(("set_free_drag", k.dtype, k.shape))
        return 0

    def raycast(self, p, v, bodyexclude, geomgroup, flg_static):
        self.calls.append(("raycast", p.shape, v.shape, p.dtype, flg_static))
        return np.zeros(p.shape[:2], np.float32), np.zeros(p.shape[:2], np.int32)

    def set_pack_spec(self, ids, lo, n):
        self.stride = self.nq + self.nv + len(ids) + 2
        return self.stride

    def get_pack(self, out=None):
        if out is None:
            return np.zeros((self.B, self.stride), np.float32)
        out[:] = 1.0
        return out


@pytest.fixture
def wrapped(quad_file):
    m = vkmujoco.load_model(quad_file)
    fake = FakeSim(6, m.nq, m.nv, m.nu)
    return vkmujoco.BatchedSim(fake, m, 6), fake


def test_step_reset_and_state_checks(wrapped):
    sim, fake = wrapped
    sim.step(np.zeros((6, 12)), 3)
    assert fake.calls[-1] == ("step", (np.float32, (6, 12)), 3)
    for bad in (np.zeros(72), np.zeros((6, 11)), np.zeros((5, 12))):
        with pytest.raises(RuntimeError):
            sim.step(bad)
    sim.reset([1, 0, 0, 1, 0, 0])
    assert fake.calls[-1] == ("reset", np.int32, (6,))
    with pytest.raises(RuntimeError):
        sim.reset(np.zeros((6, 1)))
    sim.set_state(np.zeros((6, 19)), np.zeros((6, 18)))
    assert fake.calls[-1] == ("set_state", np.float32, (6, 19), (6, 18))
    with pytest.raises(RuntimeError):
        sim.set_state(np.zeros((6, 18)), np.zeros((6, 18)))
    sim.set_env_qpos(2, np.zeros(19))
    sim.set_env_qvel(2, np.zeros(18))
    assert fake.calls[-2:] == [("set_env_state", 2, (19,), None), ("set_env_state", 2, None, (18,))]
    q, v = sim.state()
    assert q.shape == (6, 19) and v.shape == (6, 18)
    assert sim.qpos().shape == (6, 19) and sim.qvel().shape == (6, 18)
    assert sim.xpos().shape == (6, 42) and sim.cfrc_ext().shape == (6, 84) and sim.qfrc_actuator().shape == (6, 18)
    assert sim.sensordata().shape == (6, 0)


def test_env_params_and_drag_checks(wrapped):
    sim, fake = wrapped
    sim.set_env_params(mass_scale=np.ones((6, 14)), com_delta=np.zeros((6, 14, 3)), friction_scale=np.ones(6), gain_scale=np.ones((6, 12)))
    assert fake.calls[-1] == ("set_env_params", None, True, True)
    sim.set_env_params(env_idx=[1, 3], mass_scale=np.ones((2, 14)))
    assert fake.calls[-1][1] == np.int32
    for kw in ({"mass_scale": np.ones((6, 13))}, {"com_delta": np.zeros((6, 14))}, {"friction_scale": np.ones((6, 1))},
               {"gain_scale": np.ones((5, 12))}):
        with pytest.raises(RuntimeError):
            sim.set_env_params(**kw)
    assert sim.num_free_joints() == 1
    sim.set_free_drag(np.ones((6, 1)))
    assert fake.calls[-1] == ("set_free_drag", np.float32, (6, 1))
    with pytest.raises(RuntimeError):
        sim.set_free_drag(np.ones(6))
    fake.set_env_params = lambda *a, **k: -1
    with pytest.raises(RuntimeError):
        sim.set_env_params(friction_scale=np.ones(6))


def test_raycast_broadcast_and_checks(wrapped):
    sim, fake = wrapped
    dist, gid = sim.raycast(np.zeros((5, 3)), np.tile([0, 0, -1.0], (5, 1)))
    assert fake.calls[-1] == ("raycast", (6, 5, 3), (6, 5, 3), np.float32, 1)
    assert dist.shape == (6, 5) and gid.dtype == np.int32
    sim.raycast(np.zeros((6, 4, 3)), np.zeros((4, 3)), flg_static=False)
    assert fake.calls[-1][-1] == 0
    for p, v in ((np.zeros((6, 4, 2)), np.zeros((4, 3))), (np.zeros((4, 3)), np.zeros((5, 3))), (np.zeros((7, 4, 3)), np.zeros((4, 3)))):
        with pytest.raises(RuntimeError):
            sim.raycast(p, v)
    with pytest.raises(RuntimeError):
        sim.raycast(np.zeros((4, 3)), np.zeros((4, 3)), geomgroup=[1, 1, 1])


def test_pack_read_back(wrapped):
    sim, fake = wrapped
    with pytest.raises(RuntimeError):
        sim.read_pack()
    stride = sim.set_pack_spec([1, 4], 6, 12)
    assert stride == 19 + 18 + 4
    assert sim.read_pack().shape == (6, stride)
    out = np.zeros((6, stride), np.float32)
    sim.read_pack_into(out)
    assert np.all(out == 1.0)
    for bad in (np.zeros((6, stride)), np.zeros((6, stride + 1), np.float32), np.zeros((stride, 6), np.float32).T):
        with pytest.raises(RuntimeError):
            sim.read_pack_into(bad)
