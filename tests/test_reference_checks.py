"""Assertions of the reference's own test suite that need no MuJoCo C,
restated against the FP64 oracle (CPU only).

The reference's tests compare its engine with MuJoCo C 3.5.0, which is not
installed here.  Beside those comparisons they assert facts that hold for any
correct implementation of the step: a free body in zero gravity keeps its
velocity, a floating ball has no constraint rows, each violated limit adds a
row, gravity compensation on a hanging chain is zero, a body with full
gravity compensation hovers, frictionloss adds one row per dof and slows the
joint, an excluded body pair yields no pair and no contact, a joint
equality adds one row, the implicit integrators differ from Euler where the
velocity derivative of an actuator matters, identity per-env parameters
change nothing, an explicit pair collides geoms that filtering skips and
sets the contact's friction, a spherical ellipsoid behaves as a sphere, and
every primitive dropped on the floor is caught.  Each test names the reference test it follows (file:line
within the reference's tests/ folder) and, where the mechanics allow,
replaces the reference's loose bound with the closed-form answer.  The
models are written here, in the spirit of the reference's, not copied.
"""
import ctypes as C

import numpy as np
import pytest

import mjb200
import oracle

G = 9.81


def env_from_xml(xml, ncon_max=64, nefc_max=256):
    m = mjb200.load_model_from_string(xml)
    om = oracle.OracleModel(m.dump())
    return m, om, oracle.OracleEnv(om, ncon_max, nefc_max)


def doc(body, option='<option timestep="0.002"/>', extra=""):
    return f"<mujoco>{option}<worldbody>{body}</worldbody>{extra}</mujoco>"


FLOOR = '<geom type="plane" size="5 5 0.1"/>'


# ---------------------------------------------------------------- free bodies

def test_zero_gravity_free_body_moves_uniformly():
    """test_physics_full.cpp:572-594 (vx stays 1 to 1e-3, x reaches 0.2 to
    1e-2 after 100 steps of 2 ms): exactly, with no forces at all."""
    _, om, env = env_from_xml(doc('<body pos="0 0 0.5"><freejoint/><geom type="sphere" size="0.1" mass="1.3"/></body>',
                                  option='<option timestep="0.002" gravity="0 0 0"/>'))
    env.a["qvel"][:] = [1.0, 0, 0, 0, 0, 0]
    for _ in range(100):
        env.step()
        assert env.d.nefc == 0 and env.d.ncon == 0
    assert env.a["qvel"][0] == pytest.approx(1.0, abs=1e-14)
    assert env.a["qpos"][0] == pytest.approx(0.2, abs=1e-12)
    np.testing.assert_allclose(env.a["qpos"][1:3], [0.0, 0.5], atol=1e-14)


def test_floating_ball_has_no_constraint_rows():
    """test_physics_full.cpp:596-613: a free ball far above the floor has
    no contact and no rows."""
    _, om, env = env_from_xml(doc(FLOOR + '<body pos="0 0 10"><freejoint/><geom type="sphere" size="0.1" mass="1"/></body>'))
    env.step()
    assert env.d.ncon == 0 and env.d.nefc == 0
    assert env.a["qacc"][2] == pytest.approx(-G, rel=1e-12)


def test_slide_cart_falls_freely():
    """test_physics_full.cpp:319-341 (the z slide moves down): three
    orthogonal slides on one box give free fall along z, closed form for
    semi-implicit Euler, and nothing along x and y."""
    h = 0.002
    _, om, env = env_from_xml(doc('<body pos="0 0 1"><joint type="slide" axis="1 0 0"/><joint type="slide" axis="0 1 0"/>'
                                  '<joint type="slide" axis="0 0 1"/><geom type="box" size="0.1 0.1 0.1" mass="1"/></body>'))
    n = 50
    for _ in range(n):
        env.step()
    assert env.a["qpos"][2] == pytest.approx(-G * h * h * n * (n + 1) / 2, rel=1e-12)
    assert env.a["qvel"][2] == pytest.approx(-G * h * n, rel=1e-12)
    np.testing.assert_allclose(env.a["qpos"][:2], 0.0, atol=1e-15)


def test_ball_joint_chain_quaternions_stay_unit():
    """test_physics_full.cpp:281-317 (unit quaternion norm to 1e-3): three
    ball joints swinging for 500 steps keep unit quaternions to 1e-12."""
    _, om, env = env_from_xml(doc(
        '<body><joint type="ball"/><geom type="capsule" fromto="0 0 0 0 0 -0.4" size="0.03" mass="1"/>'
        '<body pos="0 0 -0.4"><joint type="ball"/><geom type="capsule" fromto="0 0 0 0 0 -0.4" size="0.03" mass="0.8"/>'
        '<body pos="0 0 -0.4"><joint type="ball"/><geom type="capsule" fromto="0 0 0 0 0 -0.3" size="0.03" mass="0.5"/>'
        '</body></body></body>'))
    env.a["qvel"][:] = [0.8, -1.5, 0.3, 2.0, 0.1, -0.7, -1.2, 0.9, 1.6]
    for _ in range(500):
        env.step()
    q = env.a["qpos"].reshape(3, 4)
    np.testing.assert_allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-12)
    assert np.isfinite(env.a["qvel"]).all()
    assert np.abs(q[:, 1:]).max() > 0.05   # the chain moved


# ------------------------------------------------------------- limits, springs

def test_both_violated_limits_give_limit_rows():
    """test_physics_full.cpp:615-651 (at least 2 rows with both hinge limits
    violated): exactly two limit rows, in joint order, both joints driven
    back into range, and each row's force complementary to its residual:
    f = -D min(J qacc - aref, 0).  Here the first row's push on the upper
    joint already swings the lower joint back faster than its reference
    acceleration asks, so the second row carries no force."""
    _, om, env = env_from_xml(doc(
        '<body><joint type="hinge" axis="0 1 0" limited="true" range="-0.5 0.5"/>'
        '<geom type="capsule" fromto="0 0 0 0 0 -0.5" size="0.04" mass="1"/>'
        '<body pos="0 0 -0.5"><joint type="hinge" axis="0 1 0" limited="true" range="-0.5 0.5"/>'
        '<geom type="capsule" fromto="0 0 0 0 0 -0.5" size="0.04" mass="1"/></body></body>'))
    env.a["qpos"][:] = [1.0, -1.0]
    env.step()
    e = env.efc()
    assert list(e["type"]) == [1, 1]
    # the rows' Jacobians point into the range: -1 on the upper limit of
    # joint 0, +1 on the lower limit of joint 1
    np.testing.assert_allclose(e["J"], [[-1.0, 0.0], [0.0, 1.0]], atol=1e-15)
    jar = e["J"] @ env.a["qacc"] - e["aref"]
    np.testing.assert_allclose(e["force"], -e["D"] * np.minimum(jar, 0.0), rtol=1e-9, atol=1e-9 * np.abs(e["force"]).max())
    assert e["force"][0] > 0 and e["force"][1] >= 0
    # both joints are driven back towards their ranges
    assert env.a["qacc"][0] < 0 < env.a["qacc"][1]


def test_damped_springs_lose_amplitude():
    """test_physics_full.cpp:653-700 (2000 steps bounded, late amplitude
    below early): two independent damped hinge springs started at +1 and -1
    rad; after 4 s the amplitude has decayed by more than 10x."""
    _, om, env = env_from_xml(doc(
        '<body><joint type="hinge" axis="0 1 0" stiffness="12" damping="0.6"/>'
        '<geom type="capsule" fromto="0 0 0 0 0 -0.5" size="0.04" mass="1"/></body>'
        '<body pos="1 0 0"><joint type="hinge" axis="0 1 0" stiffness="6" damping="0.4"/>'
        '<geom type="capsule" fromto="0 0 0 0 0 -0.5" size="0.04" mass="1"/></body>'))
    env.a["qpos"][:] = [1.0, -1.0]
    early = late = 0.0
    for i in range(2000):
        env.step()
        a = np.abs(env.a["qpos"]).max()
        assert np.isfinite(env.a["qpos"]).all() and a < 20
        if i < 100:
            early = max(early, a)
        if i >= 1900:
            late = max(late, a)
    assert late < 0.1 * early


# ------------------------------------------------------- gravity compensation

_HANGING = ('<body gravcomp="{g}"><joint type="hinge" axis="0 1 0"/><geom type="capsule" fromto="0 0 0 0 0 -0.4" size="0.03" mass="1"/>'
            '<body gravcomp="{g}" pos="0 0 -0.4"><joint type="hinge" axis="1 0 0"/>'
            '<geom type="capsule" fromto="0 0 0 0 0 -0.3" size="0.03" mass="0.7"/></body></body>')


def test_zero_gravcomp_adds_no_force():
    """test_gravcomp.cpp:122-128: gravcomp = 0 adds nothing (no springs or
    dampers either, so the passive force is zero everywhere)."""
    _, om, env = env_from_xml(doc(_HANGING.format(g=0)))
    env.a["qpos"][:] = [0.4, -0.9]
    env.step()
    np.testing.assert_array_equal(env.a["qfrc_passive"], 0.0)


def test_hanging_chain_gravcomp_is_zero_at_rest():
    """test_gravcomp.cpp:299-319: a chain hanging straight down has zero
    gravity torque about its hinges, so full compensation is zero there;
    displaced, it equals minus the gravity torque."""
    _, om, env = env_from_xml(doc(_HANGING.format(g=1)))
    env.step()
    np.testing.assert_allclose(env.a["qfrc_passive"], 0.0, atol=1e-12)
    _, om0, env0 = env_from_xml(doc(_HANGING.format(g=0)))
    for e in (env, env0):
        e.a["qpos"][:] = [0.4, -0.9]
        e.a["qvel"][:] = 0
        e.step()
    # gravity's generalized force is -qfrc_bias at zero velocity
    np.testing.assert_allclose(env.a["qfrc_passive"], env0.a["qfrc_bias"], rtol=1e-10)
    assert np.abs(env.a["qfrc_passive"]).min() > 0.1


def test_full_gravcomp_free_body_hovers():
    """test_gravcomp.cpp:263-289 (z stays within 0.1 of 2.0 over 100 steps):
    full compensation of a free body cancels gravity exactly."""
    _, om, env = env_from_xml(doc('<body pos="0 0 2" gravcomp="1"><freejoint/><geom type="box" size="0.1 0.2 0.15" mass="2.5"/></body>'))
    for _ in range(100):
        env.step()
    np.testing.assert_allclose(env.a["qpos"][:3], [0, 0, 2.0], atol=1e-12)
    np.testing.assert_allclose(env.a["qvel"], 0.0, atol=1e-12)


# ------------------------------------------------------------------ cfrc_ext

def test_cfrc_ext_zero_without_contacts_then_set_on_impact():
    """test_cfrc_ext.cpp:102-112 (zero with no contacts), 163-194 (non-zero
    once a falling ball touches the floor) and 286-292 (nbody x 6)."""
    _, om, env = env_from_xml(doc(FLOOR + '<body pos="0 0 0.13"><freejoint/><geom type="sphere" size="0.1" mass="1"/></body>'))
    assert env.a["cfrc_ext"].size == om.nbody * 6
    touched = None
    for i in range(200):
        env.step()
        if env.d.ncon == 0:
            assert touched is None
            np.testing.assert_array_equal(env.a["cfrc_ext"], 0.0)
        elif touched is None:
            touched = i
    assert touched is not None
    cf = env.a["cfrc_ext"].reshape(om.nbody, 6)
    assert cf[1, 5] > 0                      # the floor pushes the ball up
    assert np.isfinite(cf).all()


# ------------------------------------------------------------- frictionloss

def test_frictionloss_rows_one_per_dof():
    """test_dof_friction.cpp:109-150: one row per dof with frictionloss,
    none for dofs without, and no equality rows."""
    _, om, env = env_from_xml(doc('<body><joint type="hinge" axis="0 1 0" frictionloss="0.5"/>'
                                  '<geom type="capsule" fromto="0 0 0 0 0 -0.5" size="0.03" mass="1"/></body>'))
    env.a["qvel"][0] = 0.3
    env.step()
    assert list(env.efc()["type"]) == [0]
    _, om, env = env_from_xml(doc(
        '<body><joint type="hinge" axis="0 1 0" frictionloss="0.5"/><geom type="capsule" fromto="0 0 0 0 0 -0.4" size="0.03" mass="1"/>'
        '<body pos="0 0 -0.4"><joint type="hinge" axis="0 1 0"/><geom type="capsule" fromto="0 0 0 0 0 -0.4" size="0.03" mass="1"/>'
        '<body pos="0 0 -0.4"><joint type="hinge" axis="1 0 0"/><geom type="capsule" fromto="0 0 0 0 0 -0.3" size="0.03" mass="1"/>'
        '</body></body></body>'))
    env.a["qpos"][:] = [0.2, -0.3, 0.1]
    env.step()
    e = env.efc()
    assert list(e["type"]) == [0]
    np.testing.assert_allclose(e["J"], [[1.0, 0.0, 0.0]], atol=1e-15)


def test_frictionloss_decelerates_at_f_over_m():
    """test_dof_friction.cpp:327-355 (|v| below its start of 5 after 100
    steps): a horizontal slide started at 5 m/s.  While it slides, the
    friction row sits in the saturated zone of its cost, its force is
    exactly -frictionloss, and the speed falls by h f / m per step."""
    h, m, f = 0.002, 2.0, 6.0
    _, om, env = env_from_xml(doc(f'<body><joint type="slide" axis="1 0 0" frictionloss="{f}"/>'
                                  f'<geom type="box" size="0.1 0.1 0.1" mass="{m}"/></body>'))
    env.a["qvel"][0] = 5.0
    for n in range(1, 101):
        env.step()
        assert env.a["qvel"][0] == pytest.approx(5.0 - n * h * f / m, abs=1e-9)
        assert env.efc()["force"][0] == pytest.approx(-f, abs=1e-9)
    assert abs(env.a["qvel"][0]) < 5.0


def test_joint_equality_and_frictionloss_rows():
    """test_equality.cpp:247-263 (a joint equality gives one row) and
    test_dof_friction.cpp:289-309 (equality and friction rows together):
    the equality row comes first, then the friction row."""
    body = ('<body><joint name="a" type="hinge" axis="0 1 0" frictionloss="0.2"/>'
            '<geom type="capsule" fromto="0 0 0 0.4 0 0" size="0.03" mass="1"/></body>'
            '<body pos="0 0.5 0"><joint name="b" type="hinge" axis="0 1 0"/>'
            '<geom type="capsule" fromto="0 0 0 0.4 0 0" size="0.03" mass="1"/></body>')
    _, om, env = env_from_xml(doc(body, extra='<equality><joint joint1="a" joint2="b"/></equality>'))
    env.a["qpos"][:] = [0.3, 0.1]
    env.step()
    e = env.efc()
    assert list(e["type"]) == [5, 0]
    # the equality row constrains q_a - q_b (polynomial coefficient 1)
    np.testing.assert_allclose(e["J"][0], [1.0, -1.0], atol=1e-15)


# -------------------------------------------------------------------- exclude

_ARMS = ('<body name="torso" pos="0 0 0.6"><freejoint/><geom type="capsule" size="0.1 0.15" mass="5"/>'
         '<body name="arm" pos="0.2 0 0.15"><joint type="hinge" axis="0 1 0"/><geom type="capsule" size="0.05 0.15" mass="1"/>'
         '<body name="hand" pos="0 0 -0.3"><joint type="hinge" axis="0 1 0"/><geom type="capsule" size="0.04 0.12" mass="0.5"/></body></body>'
         '<body name="leg" pos="0 0 -0.15"><joint type="hinge" axis="0 1 0"/><geom type="capsule" size="0.06 0.2" mass="2"/>'
         '<body name="foot" pos="0 0 -0.4"><joint type="hinge" axis="0 1 0"/><geom type="capsule" size="0.05 0.15" mass="1"/></body></body>'
         '</body>')


def test_exclude_removes_exactly_one_pair():
    """test_exclude.cpp:71-131: a model with one exclude has exactly one
    candidate pair fewer than the same model without it."""
    m0 = mjb200.load_model_from_string(doc(FLOOR + _ARMS))
    m1 = mjb200.load_model_from_string(doc(FLOOR + _ARMS, extra='<contact><exclude body1="torso" body2="foot"/></contact>'))
    n0 = int(m0.dump()["sizes"][7])
    n1 = int(m1.dump()["sizes"][7])
    assert n0 > 0 and n1 == n0 - 1


def test_excluded_overlapping_bodies_do_not_collide():
    """test_exclude.cpp:181-220: two overlapping free spheres collide, unless
    their bodies are excluded."""
    spheres = ('<body name="A" pos="0 0 0.5"><freejoint/><geom type="sphere" size="0.2" mass="1"/></body>'
               '<body name="B" pos="0.1 0 0.5"><freejoint/><geom type="sphere" size="0.2" mass="1"/></body>')
    _, om, env = env_from_xml(doc(spheres))
    env.step()
    assert env.d.ncon > 0
    _, om, env = env_from_xml(doc(spheres, extra='<contact><exclude body1="A" body2="B"/></contact>'))
    assert int(om.dump["sizes"][7]) == 0
    env.step()
    assert env.d.ncon == 0 and env.d.nefc == 0


# -------------------------------------------------------------- integrators

@pytest.mark.parametrize("integrator,code", [("implicitfast", 3), ("implicit", 2)])
def test_implicit_integrators_fold_the_velocity_actuator(integrator, code):
    """test_implicit.cpp:296-335 (implicit and Euler differ by more than 1e-3
    on a stiff system): a slide driven by a velocity servo of gain kv at
    ctrl 0.  Euler treats the servo force -kv v explicitly; the implicit
    integrators fold its velocity derivative into the mass:
        Euler:    v1 = v0 + h (-kv v0 - m g) / m
        implicit: v1 = v0 + h (-kv v0 - m g) / (m + h kv)."""
    h, m, kv, v0 = 0.005, 1.5, 400.0, 1.0
    body = (f'<body pos="0 0 2"><joint name="s" type="slide" axis="0 0 1"/><geom type="sphere" size="0.08" mass="{m}"/></body>')
    act = f'<actuator><velocity joint="s" kv="{kv}"/></actuator>'
    out = {}
    for integ in ("Euler", integrator):
        model, om, env = env_from_xml(doc(body, option=f'<option timestep="{h}" integrator="{integ}"/>', extra=act))
        if integ != "Euler":
            assert int(model.dump()["opt_int"][3]) == code
        env.a["qvel"][0] = v0
        env.step()
        out[integ] = env.a["qvel"][0]
    f = -kv * v0 - m * G
    assert out["Euler"] == pytest.approx(v0 + h * f / m, rel=1e-12)
    assert out[integrator] == pytest.approx(v0 + h * f / (m + h * kv), rel=1e-12)
    assert abs(out[integrator] - out["Euler"]) > 1e-3


# ------------------------------------------------------------- per-env params

_RAND_SCENE = (FLOOR + '<body pos="0 0 0.1"><freejoint/><geom type="box" size="0.1 0.1 0.1" mass="1" friction="0.6"/></body>'
               '<body pos="1 0 1"><joint name="h" type="hinge" axis="0 1 0"/>'
               '<geom type="capsule" fromto="0 0 0 0.4 0 0" size="0.03" mass="1"/></body>')
_RAND_ACT = '<actuator><motor joint="h" gear="2"/></actuator>'


def _rand_rollout(mass=None, friction=1.0, gain=None, com=None, steps=60):
    _, om, env = env_from_xml(doc(_RAND_SCENE, extra=_RAND_ACT))
    env.a["qvel"][0] = 1.5
    env.a["ctrl"][0] = 0.7
    keep = []

    def arr(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, np.float64)
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_double))

    rand = oracle.ORand(arr(mass), friction, arr(gain), arr(com), None) if any(x is not None for x in (mass, gain, com)) or friction != 1.0 else None
    for _ in range(steps):
        env.step(0, rand)
    return env.a["qpos"].copy(), env.a["qvel"].copy()


def test_identity_env_params_change_nothing():
    """test_env_rand.cpp:114-117: identity parameters (unit scales, zero COM
    offset) step exactly like the non-randomised path."""
    q0, v0 = _rand_rollout()
    q1, v1 = _rand_rollout(mass=np.ones(3), friction=1.0, gain=np.ones(1), com=np.zeros(9))
    np.testing.assert_array_equal(q0, q1)
    np.testing.assert_array_equal(v0, v1)


def test_env_params_change_the_result():
    """test_env_rand.cpp:121-126: a mass scale changes the arm's swing, a
    friction scale changes the box's slide, an actuator gain scale changes
    the driven arm."""
    q0, _ = _rand_rollout()
    qm, _ = _rand_rollout(mass=[1.0, 1.0, 1.3])
    qf, _ = _rand_rollout(friction=0.4)
    qg, _ = _rand_rollout(gain=[1.5])
    assert np.abs(qm[7] - q0[7]) > 1e-3      # arm hinge
    assert np.abs(qm[:3] - q0[:3]).max() < 1e-12   # the box does not see the arm's mass
    assert np.abs(qf[0] - q0[0]) > 1e-3      # box slide along x
    assert np.abs(qg[7] - q0[7]) > 1e-3


# ------------------------------------------------------------------ collision

# contact record fields (oracle layout): pos 0-2, frame 3-11, dist 12,
# pair 13, geom1 14, geom2 15, condim 16, mu0 17
_DIST, _G1, _G2, _MU0 = 12, 14, 15, 17


def test_explicit_pair_collides_geoms_that_filtering_skips():
    """test_collision_full.cpp:114-122 and 142-150: a geom with contype =
    conaffinity = 0 gets no pair and no contact, unless an explicit <pair>
    names it; then it touches the floor, 1 cm deep as placed."""
    scene = ('<geom name="floor" type="plane" size="5 5 0.1"/><body pos="0 0 0.09"><freejoint/>'
             '<geom name="ball" type="sphere" size="0.1" mass="1" contype="0" conaffinity="0"/></body>')
    _, om, env = env_from_xml(doc(scene))
    assert om.npair == 0
    env.step()
    assert env.d.ncon == 0
    _, om, env = env_from_xml(doc(scene, extra='<contact><pair geom1="ball" geom2="floor"/></contact>'))
    assert om.npair == 1
    env.step()
    assert env.d.ncon == 1
    c = env.contacts()[0]
    assert c[_DIST] == pytest.approx(-0.01, abs=1e-12)
    assert sorted((int(c[_G1]), int(c[_G2]))) == [0, 1]


def test_explicit_pair_friction_sets_the_contact_friction():
    """test_collision_full.cpp:170-178 (pairs with friction 0.5 and 2.0
    produce contacts): each contact carries its pair's friction, and the
    box on the low-friction pair slides farther."""
    scene = ('<geom name="floor" type="plane" size="5 5 0.1" contype="0" conaffinity="0"/>'
             '<body pos="0 0 0.099"><freejoint/><geom name="a" type="box" size="0.1 0.1 0.1" mass="1" contype="0" conaffinity="0"/></body>'
             '<body pos="0 1 0.099"><freejoint/><geom name="b" type="box" size="0.1 0.1 0.1" mass="1" contype="0" conaffinity="0"/></body>')
    pairs = ('<contact><pair geom1="a" geom2="floor" friction="0.5 0.5 0.005 0.0001 0.0001"/>'
             '<pair geom1="b" geom2="floor" friction="2.0 2.0 0.005 0.0001 0.0001"/></contact>')
    _, om, env = env_from_xml(doc(scene, extra=pairs))
    env.a["qvel"][0] = 1.0
    env.a["qvel"][6] = 1.0
    env.step()
    mu = {}
    for c in env.contacts():
        g = max(int(c[_G1]), int(c[_G2]))
        mu.setdefault(g, set()).add(round(float(c[_MU0]), 12))
    assert mu == {1: {0.5}, 2: {2.0}}
    for _ in range(150):
        env.step()
    xa, xb = env.a["qpos"][0], env.a["qpos"][7]
    assert xa > xb + 0.02 and xb > 0


def test_spherical_ellipsoid_matches_sphere():
    """test_collision_ellipsoid.cpp:177-199 (an ellipsoid with three equal
    radii stays within 1 of a sphere): a tumbling ellipsoid with equal radii
    and a sphere of the same mass bounce on the floor identically, to
    1e-9 over 300 steps."""
    out = []
    for g in ('type="sphere" size="0.1"', 'type="ellipsoid" size="0.1 0.1 0.1"'):
        _, om, env = env_from_xml(doc(FLOOR + f'<body pos="0 0 0.2"><freejoint/><geom {g} mass="1.2"/></body>'))
        env.a["qvel"][:] = [0.5, -0.2, -1.0, 3.0, -2.0, 1.0]
        hist = []
        for _ in range(300):
            env.step()
            hist.append(np.concatenate([env.a["qpos"], env.a["qvel"], [env.d.ncon]]))
        out.append(np.array(hist))
    assert out[0][:, -1].max() == 1
    np.testing.assert_allclose(out[1], out[0], atol=1e-9)


@pytest.mark.parametrize("geom", ['type="sphere" size="0.1"', 'type="capsule" size="0.06 0.12"', 'type="box" size="0.1 0.08 0.06"',
                                  'type="ellipsoid" size="0.12 0.08 0.06"', 'type="cylinder" size="0.08 0.1"'])
def test_dropped_primitive_is_caught(geom):
    """test_batched_collision_primitives.cpp:111-124 (each primitive dropped
    on the floor stays within |qpos| < 2 after 200 steps) and
    test_collision_full.cpp:221-232 (no fall through): tilted, dropped from
    0.4 m, the body hits the floor at about 2.8 m/s, sinks less than 3 cm
    into it on impact (the soft contact's default 20 ms time constant) and
    then stays on it: in contact and below 0.2 m for each of the last 300
    of 1500 steps, less than 1 cm deep.  (The sphere, capsule and box come
    to rest; the ellipsoid keeps rocking and the cylinder rolls on its
    side, as condim 3 models no rolling friction.)"""
    _, om, env = env_from_xml(doc(FLOOR + f'<body pos="0 0 0.4" euler="20 35 0"><freejoint/><geom {geom} mass="1"/></body>'))
    lowest = np.inf
    for i in range(1500):
        env.step()
        cs = env.contacts()
        for c in cs:
            lowest = min(lowest, c[_DIST])
        if i >= 1200:
            assert len(cs) >= 1 and cs[:, _DIST].min() > -0.01
            assert 0 < env.a["qpos"][2] < 0.2
    assert lowest > -0.03
    assert np.isfinite(env.a["qpos"]).all() and np.isfinite(env.a["qvel"]).all()


@pytest.mark.parametrize("eulerdamp", [True, False])
def test_euler_folds_joint_damping_unless_disabled(eulerdamp):
    """test_implicit.cpp:199-223 (damped pendulum): MuJoCo's Euler
    integrator puts the joint damping d on the mass matrix's diagonal,
    v1 = v0 + h (-d v0) / (m + h d); with the eulerdamp flag disabled the
    damping force is explicit, v1 = v0 + h (-d v0) / m.  A horizontal slide
    with no gravity along it."""
    h, m, d, v0 = 0.01, 0.5, 40.0, 2.0
    flag = "" if eulerdamp else '<flag eulerdamp="disable"/>'
    _, om, env = env_from_xml(doc(f'<body><joint type="slide" axis="1 0 0" damping="{d}"/><geom type="box" size="0.1 0.1 0.1" mass="{m}"/></body>',
                                  option=f'<option timestep="{h}">{flag}</option>'))
    env.a["qvel"][0] = v0
    env.step()
    want = v0 + h * (-d * v0) / (m + h * d) if eulerdamp else v0 + h * (-d * v0) / m
    assert env.a["qvel"][0] == pytest.approx(want, rel=1e-12)
