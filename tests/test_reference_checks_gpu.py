"""The closed-form answers of test_reference_checks.py, through the CUDA
engine (FP32, C ABI).

The CPU file pins the FP64 oracle to assertions of the reference's own tests
that need no MuJoCo C; here the engine meets the same answers, with FP32
tolerances written in each test: uniform motion in zero gravity,
frictionloss deceleration at exactly f / m, the implicit integrators'
velocity-servo fold, a hovering fully compensated body, excluded bodies,
a spherical ellipsoid against a sphere, primitives caught by the floor and
identity per-env parameters.
"""
import numpy as np
import pytest

import mjb200
from test_reference_checks import FLOOR, _RAND_ACT, _RAND_SCENE, G, doc

pytestmark = pytest.mark.gpu

B = 4


def sim_from_xml(xml, nenv=B, **kw):
    model = mjb200.load_model_from_string(xml)
    return model, mjb200.BatchedSim(model, nenv, **kw)


def test_gpu_zero_gravity_free_body_moves_uniformly():
    """test_physics_full.cpp:572-594: vx stays 1, x advances by 0.2 in 100
    steps of 2 ms (one fused launch of 100 substeps)."""
    model, sim = sim_from_xml(doc('<body pos="0 0 0.5"><freejoint/><geom type="sphere" size="0.1" mass="1.3"/></body>',
                                  option='<option timestep="0.002" gravity="0 0 0"/>'))
    q0 = np.tile([0, 0, 0.5, 1, 0, 0, 0], (B, 1)).astype(np.float32)
    v0 = np.tile([1, 0, 0, 0, 0, 0], (B, 1)).astype(np.float32)
    sim.set_state(q0, v0)
    sim.step(None, 100)
    q, v = sim.state()
    st = sim.stats()
    assert np.all(st["ncon"] == 0) and np.all(st["nefc"] == 0) and np.all(st["status"] == 0)
    np.testing.assert_allclose(v, v0, atol=1e-6)
    np.testing.assert_allclose(q[:, 0], 0.2, atol=1e-5)
    np.testing.assert_allclose(q[:, 1:], q0[:, 1:], atol=1e-7)
    sim.close()


def test_gpu_frictionloss_decelerates_at_f_over_m():
    """test_dof_friction.cpp:327-355: a horizontal slide started at 5 m/s
    loses h f / m of speed per step while it slides (the friction row is
    saturated at -f)."""
    h, m, f = 0.002, 2.0, 6.0
    model, sim = sim_from_xml(doc(f'<body><joint type="slide" axis="1 0 0" frictionloss="{f}"/>'
                                  f'<geom type="box" size="0.1 0.1 0.1" mass="{m}"/></body>'))
    sim.set_state(np.zeros((B, 1), np.float32), np.full((B, 1), 5.0, np.float32))
    n = 0
    for k in (1, 9, 90):
        sim.step(None, k)
        n += k
        _, v = sim.state()
        np.testing.assert_allclose(v[:, 0], 5.0 - n * h * f / m, atol=2e-5)
        st = sim.stats()
        assert np.all(st["nefc"] == 1) and np.all(st["status"] == 0)
    sim.close()


@pytest.mark.parametrize("integrator,code", [("implicitfast", 3), ("implicit", 2)])
def test_gpu_implicit_integrators_fold_the_velocity_actuator(integrator, code):
    """test_implicit.cpp:296-335: a slide driven by a velocity servo (gain
    kv, ctrl 0) steps to v0 + h (-kv v0 - m g) / m under Euler and to
    v0 + h (-kv v0 - m g) / (m + h kv) under the implicit integrators."""
    h, m, kv, v0 = 0.005, 1.5, 400.0, 1.0
    body = f'<body pos="0 0 2"><joint name="s" type="slide" axis="0 0 1"/><geom type="sphere" size="0.08" mass="{m}"/></body>'
    act = f'<actuator><velocity joint="s" kv="{kv}"/></actuator>'
    f = -kv * v0 - m * G
    want = {"Euler": v0 + h * f / m, integrator: v0 + h * f / (m + h * kv)}
    for integ, icode in (("Euler", 0), (integrator, code)):
        model, sim = sim_from_xml(doc(body, option=f'<option timestep="{h}" integrator="{integ}"/>', extra=act), integrator=icode)
        sim.set_state(np.zeros((B, 1), np.float32), np.full((B, 1), v0, np.float32))
        sim.step(np.zeros((B, 1), np.float32), 1)
        _, v = sim.state()
        np.testing.assert_allclose(v[:, 0], want[integ], rtol=1e-5)
        sim.close()
    assert abs(want[integrator] - want["Euler"]) > 1e-3


def test_gpu_full_gravcomp_free_body_hovers():
    """test_gravcomp.cpp:263-289: full compensation of a free body cancels
    gravity; after 100 steps it has not moved."""
    model, sim = sim_from_xml(doc('<body pos="0 0 2" gravcomp="1"><freejoint/><geom type="box" size="0.1 0.2 0.15" mass="2.5"/></body>'))
    q0 = np.tile([0, 0, 2.0, 1, 0, 0, 0], (B, 1)).astype(np.float32)
    sim.set_state(q0, np.zeros((B, 6), np.float32))
    sim.step(None, 100)
    q, v = sim.state()
    np.testing.assert_allclose(q, q0, atol=1e-5)
    np.testing.assert_allclose(v, 0.0, atol=1e-5)
    sim.close()


def test_gpu_excluded_overlapping_bodies_do_not_collide():
    """test_exclude.cpp:181-220: overlapping free spheres collide unless
    their bodies are excluded."""
    spheres = ('<body name="A" pos="0 0 0.5"><freejoint/><geom type="sphere" size="0.2" mass="1"/></body>'
               '<body name="B" pos="0.1 0 0.5"><freejoint/><geom type="sphere" size="0.2" mass="1"/></body>')
    for extra, collide in (("", True), ('<contact><exclude body1="A" body2="B"/></contact>', False)):
        model, sim = sim_from_xml(doc(spheres, extra=extra))
        sim.step(None, 1)
        st = sim.stats()
        assert np.all(st["status"] == 0)
        assert np.all(st["ncon"] > 0) if collide else np.all(st["ncon"] == 0) and np.all(st["nefc"] == 0)
        sim.close()


def test_gpu_spherical_ellipsoid_matches_sphere():
    """test_collision_ellipsoid.cpp:177-199: an ellipsoid with equal radii
    and a sphere of the same mass, tumbling onto the floor, follow the same
    path (FP32, 200 steps, through first contact)."""
    out = []
    for g in ('type="sphere" size="0.1"', 'type="ellipsoid" size="0.1 0.1 0.1"'):
        model, sim = sim_from_xml(doc(FLOOR + f'<body pos="0 0 0.2"><freejoint/><geom {g} mass="1.2"/></body>'))
        sim.set_state(np.tile([0, 0, 0.2, 1, 0, 0, 0], (B, 1)).astype(np.float32),
                      np.tile([0.5, -0.2, -1.0, 3.0, -2.0, 1.0], (B, 1)).astype(np.float32))
        ncon = 0
        for _ in range(20):
            sim.step(None, 10)
            ncon = max(ncon, int(sim.stats()["ncon"].max()))
        q, v = sim.state()
        out.append((q, v, ncon))
        sim.close()
    assert out[0][2] == 1 and out[1][2] == 1
    np.testing.assert_allclose(out[1][0], out[0][0], atol=1e-4)
    np.testing.assert_allclose(out[1][1], out[0][1], atol=1e-3)


@pytest.mark.parametrize("geom", ['type="sphere" size="0.1"', 'type="capsule" size="0.06 0.12"', 'type="box" size="0.1 0.08 0.06"',
                                  'type="ellipsoid" size="0.12 0.08 0.06"', 'type="cylinder" size="0.08 0.1"'])
def test_gpu_dropped_primitive_is_caught(geom):
    """test_batched_collision_primitives.cpp:111-124: dropped tilted from
    0.4 m, each primitive is on the floor (in contact, below 0.2 m) after
    1500 steps."""
    model, sim = sim_from_xml(doc(FLOOR + f'<body pos="0 0 0.4" euler="20 35 0"><freejoint/><geom {geom} mass="1"/></body>'))
    sim.step(None, 1500)
    q, v = sim.state()
    st = sim.stats()
    assert np.isfinite(q).all() and np.isfinite(v).all()
    assert np.all(st["status"] == 0) and np.all(st["ncon"] >= 1)
    assert np.all((q[:, 2] > 0) & (q[:, 2] < 0.2))
    sim.close()


def test_gpu_identity_env_params_change_nothing():
    """test_env_rand.cpp:114-117: a sim with per-env parameters set to the
    identity (unit mass, friction and gain scales, zero COM offsets) steps
    like the sim without randomisation (the reference allows 1e-6)."""
    model = mjb200.load_model_from_string(doc(_RAND_SCENE, extra=_RAND_ACT))
    nb, nu = model.dump()["sizes"][3], model.nu
    runs = []
    for rand in (0, 1):
        sim = mjb200.BatchedSim(model, B, domain_rand=rand)
        if rand:
            assert sim.set_env_params(mass_scale=np.ones((B, nb)), friction_scale=np.ones(B), gain_scale=np.ones((B, nu)),
                                      com_delta=np.zeros((B, nb, 3))) == 0
        q0, v0 = sim.state()
        v0[:, 0] = 1.5
        sim.set_state(q0, v0)
        for _ in range(3):
            sim.step(np.full((B, nu), 0.7, np.float32), 20)
        runs.append(sim.state())
        sim.close()
    np.testing.assert_allclose(runs[1][0], runs[0][0], atol=1e-6)
    np.testing.assert_allclose(runs[1][1], runs[0][1], atol=1e-6)
