"""Known answers and structural rules that pin the FP64 oracle (CPU only).

MuJoCo C is not installed here and the reference ships no golden vectors for
this path, so the oracle is pinned by closed-form mechanics (free fall, a
pendulum, rigid-body mass matrices, exp-map rotation), by the reference's own
structural rules (condim 3 pyramidal contacts give 4 rows each,
tests/test_friction_condim3.cpp:88-101 of the reference) and by the
optimality conditions of the Gauss-principle problem the Newton solver
minimises (solver.hpp:592-854 of the reference).
"""
import numpy as np
import pytest

import mjb200
import oracle

G = 9.81
H = 0.005


def env_from_xml(xml, ncon_max=64, nefc_max=256):
    m = mjb200.load_model_from_string(xml)
    om = oracle.OracleModel(m.dump())
    return om, oracle.OracleEnv(om, ncon_max, nefc_max)


def wrap(body, option='<option timestep="0.005"/>', extra=""):
    return f"<mujoco>{option}{extra}<worldbody>{body}</worldbody></mujoco>"


PLANE = '<geom type="plane" size="5 5 0.1"/>'


def test_free_fall_closed_form():
    om, env = env_from_xml(wrap(PLANE + '<body pos="0 0 1"><freejoint/><geom type="sphere" size="0.1" mass="2"/></body>'))
    for n in range(1, 11):
        env.step()
        # semi-implicit Euler: v_n = -g h n, z_n = 1 - g h^2 n (n + 1) / 2
        assert env.a["qvel"][2] == pytest.approx(-G * H * n, rel=1e-12)
        assert env.a["qpos"][2] == pytest.approx(1 - G * H * H * n * (n + 1) / 2, rel=1e-12)
        assert env.d.ncon == 0 and env.d.nefc == 0 and env.d.status == 0
    np.testing.assert_allclose(env.a["qpos"][3:], [1, 0, 0, 0], atol=1e-15)


@pytest.mark.parametrize("theta", [0.3, -1.1, 2.0])
def test_pendulum_acceleration(theta):
    L, m, r = 0.7, 1.5, 0.02
    om, env = env_from_xml(wrap(f'<body><joint type="hinge" axis="0 1 0"/><geom type="sphere" pos="0 0 {-L}" size="{r}" mass="{m}"/></body>'))
    env.a["qpos"][0] = theta
    env.step()
    inertia = m * L * L + 0.4 * m * r * r
    want = -m * G * L * np.sin(theta) / inertia
    assert env.a["qacc_smooth"][0] == pytest.approx(want, rel=1e-10)
    assert env.a["M"][0] == pytest.approx(inertia, rel=1e-10)


def test_free_box_mass_matrix_and_invweights():
    m_, hx, hy, hz = 3.0, 0.1, 0.2, 0.3
    xml = wrap(f'<body pos="0 0 2" quat="0.9 0.1 0.3 0.2"><freejoint/><geom type="box" size="{hx} {hy} {hz}" mass="{m_}"/></body>')
    model = mjb200.load_model_from_string(xml)
    d = model.dump()
    om = oracle.OracleModel(d)
    env = oracle.OracleEnv(om)
    env.step()
    I = m_ / 3 * np.array([hy * hy + hz * hz, hx * hx + hz * hz, hx * hx + hy * hy])
    M = env.a["M"].reshape(6, 6)
    # translational dofs in the world frame, rotational dofs in the body frame
    np.testing.assert_allclose(M, np.diag([m_, m_, m_, *I]), atol=1e-12)
    np.testing.assert_allclose(d["dof_invweight0"], [1 / m_] * 3 + [np.mean(1 / I)] * 3, rtol=1e-10)
    np.testing.assert_allclose(d["body_invweight0"][2:4], [1 / m_, np.mean(1 / I)], rtol=1e-10)
    assert d["opt_real"][7] == pytest.approx((3 * m_ + I.sum()) / 6, rel=1e-12)  # meaninertia


def test_exp_map_rotation():
    om, env = env_from_xml(wrap('<body pos="0 0 3"><freejoint/><geom type="sphere" size="0.1" mass="1"/></body>'))
    w = np.array([0.4, -1.0, 2.0])
    env.a["qvel"][3:] = w
    env.step()
    ang = np.linalg.norm(w) * H
    ax = w / np.linalg.norm(w)
    np.testing.assert_allclose(env.a["qpos"][3:], [np.cos(ang / 2), *(np.sin(ang / 2) * ax)], atol=1e-14)
    np.testing.assert_allclose(env.a["qvel"][3:], w, atol=1e-14)  # isotropic body: no gyroscopic torque


def test_sphere_plane_contact_frame_and_rows():
    om, env = env_from_xml(wrap(PLANE + '<body pos="0 0 0.099"><freejoint/><geom type="sphere" size="0.1" mass="2"/></body>'))
    env.step()
    assert env.d.ncon == 1 and env.d.nefc == 4
    c = env.contacts()[0]
    assert c[12] == pytest.approx(-0.001, abs=1e-12)            # distance
    frame = c[3:12].reshape(3, 3)
    np.testing.assert_allclose(frame[0], [0, 0, 1], atol=1e-15)  # normal from the plane (geom 1) to the sphere
    np.testing.assert_allclose(frame @ frame.T, np.eye(3), atol=1e-14)
    np.testing.assert_allclose(c[0:3], [0, 0, -0.0005], atol=1e-12)  # midpoint of the penetration
    assert list(env.efc()["type"]) == [2, 2, 2, 2]


@pytest.mark.parametrize("geom,ncon", [
    ('<geom type="box" size="0.2 0.1 0.05" mass="1"/>', 4),
    ('<geom type="capsule" fromto="-0.2 0 0 0.2 0 0" size="0.05" mass="1"/>', 2),
    ('<geom type="sphere" size="0.05" mass="1"/>', 1),
])
def test_plane_multi_contact_counts(geom, ncon):
    om, env = env_from_xml(wrap(PLANE + f'<body pos="0 0 0.049"><freejoint/>{geom}</body>'))
    env.step()
    assert env.d.ncon == ncon
    assert env.d.nefc == 4 * ncon


def test_resting_sphere_supports_its_weight():
    m_ = 2.0
    om, env = env_from_xml(wrap(PLANE + f'<body pos="0 0 0.1"><freejoint/><geom type="sphere" size="0.1" mass="{m_}"/></body>'))
    for _ in range(600):
        env.step()
    assert env.d.ncon == 1
    assert abs(env.a["qvel"]).max() < 1e-6
    # the pyramid rows' forces sum to the normal force
    assert env.efc()["force"].sum() == pytest.approx(m_ * G, rel=1e-4)
    assert -2e-3 < env.a["qpos"][2] - 0.1 < 0
    # the contact wrench on the sphere is its weight upward through its COM,
    # and the world body takes the opposite force
    cf = env.a["cfrc_ext"].reshape(-1, 6)
    assert cf[1, 3:] == pytest.approx([0.0, 0.0, m_ * G], rel=1e-4, abs=1e-6)
    assert np.abs(cf[1, :3]).max() < 1e-9
    assert cf[0, 3:] == pytest.approx([0.0, 0.0, -m_ * G], rel=1e-4, abs=1e-6)


def test_cfrc_ext_sliding_box_friction_and_torque():
    """A resting box on a plane, then kicked sideways: at rest the contact
    wrench is the box's weight; after the kick the force is the decoded
    pyramid force sum, F = sum_c (f_n n + mu (f_0 - f_1) t1 + mu (f_2 - f_3) t2),
    with friction against the sliding direction, the torque is sum_c (p_c -
    com) x F_c about the box's COM (its subtree COM), and the world body
    takes the opposite force.  The pair's friction is the larger of the
    plane's (1.0) and the box's."""
    mu, mass = 1.0, 1.0
    xml = wrap(PLANE + '<body pos="0 0 0.05"><freejoint/><geom type="box" size="0.05 0.05 0.05" mass="%g" friction="%g 0.005 0.0001"/></body>'
               % (mass, mu))
    om, env = env_from_xml(xml)
    for _ in range(200):
        env.step()
    cf = env.a["cfrc_ext"].reshape(-1, 6)
    assert cf[1, 3:] == pytest.approx([0.0, 0.0, mass * G], rel=1e-3, abs=1e-6)
    env.a["qvel"][0] = 1.0
    env.step()
    cf = env.a["cfrc_ext"].reshape(-1, 6)
    con = env.contacts()
    assert env.d.ncon == 4
    assert cf[1, 3:] == pytest.approx(-cf[0, 3:], abs=1e-9)
    com = env.a["subtree_com"][3:6]
    efc = env.efc()
    F_sum, T = np.zeros(3), np.zeros(3)
    for c in con:
        r = int(c[19])
        f = efc["force"][r:r + 4]
        n, t1, t2 = c[3:6], c[6:9], c[9:12]
        F = f.sum() * n + mu * (f[0] - f[1]) * t1 + mu * (f[2] - f[3]) * t2
        F_sum += F
        T += np.cross(c[:3] - com, F)
    assert cf[1, 3:] == pytest.approx(F_sum, abs=1e-9)
    assert cf[1, :3] == pytest.approx(T, abs=1e-9)
    assert cf[1, 3] < -0.1 * cf[1, 5]   # friction opposes the +x slide
    assert abs(cf[1, 1]) > 1e-3         # friction below the COM tips the box about y


def test_joint_limit_and_frictionloss_rows():
    xml = wrap('<body><joint type="hinge" axis="0 1 0" range="-0.5 0.5" limited="true" frictionloss="0.1"/>'
               '<geom type="capsule" fromto="0 0 0 0 0 -0.5" size="0.02" mass="1"/></body>')
    om, env = env_from_xml(xml)
    env.a["qpos"][0] = 0.0
    env.step()
    assert list(env.efc()["type"]) == [0]                       # frictionloss row only
    env.a["qpos"][0] = 0.6
    env.a["qvel"][0] = 0.0
    env.step()
    t = list(env.efc()["type"])
    assert t == [0, 1]                                            # frictionloss before the limit row
    assert env.efc()["force"][1] > 0                               # the limit pushes back


def test_contact_overflow_keeps_first_contacts():
    om, env = env_from_xml(wrap(PLANE + '<body pos="0 0 0.049"><freejoint/><geom type="box" size="0.2 0.1 0.05" mass="1"/></body>'),
                           ncon_max=2)
    env.step()
    assert env.d.ncon == 2 and env.d.status & 4
    assert env.d.nefc == 8


def test_bad_state_resets_to_qpos0():
    om, env = env_from_xml(wrap('<body pos="0 0 1"><freejoint/><geom type="sphere" size="0.1" mass="1"/></body>'))
    env.a["qvel"][1] = np.nan
    env.step()
    assert env.d.status & 1
    assert np.isfinite(env.a["qpos"]).all() and np.isfinite(env.a["qvel"]).all()


def _gauss_residual(om, env):
    """Optimality of the Newton solution for pyramid/limit rows: with
    r = J qacc - aref and f = -D min(r, 0), M (qacc - qacc_smooth) = J^T f."""
    nv = om.nv
    M = env.a["M"].reshape(nv, nv)
    e = env.efc()
    r = e["J"] @ env.a["qacc"] - e["aref"]
    fl = env.a["efc_floss"][: len(r)]
    f = np.where(e["type"] == 5, -e["D"] * r, -e["D"] * np.minimum(r, 0.0))  # equality rows are bilateral
    f = np.where(e["type"] == 0, np.clip(-e["D"] * r, -fl, fl), f)        # frictionloss rows saturate at +-floss
    lhs = M @ (env.a["qacc"] - env.a["qacc_smooth"])
    rhs = e["J"].T @ f
    return np.linalg.norm(lhs - rhs) / max(np.linalg.norm(M @ env.a["qacc_smooth"]), 1.0), f, e["force"]


def test_newton_solution_is_gauss_optimal_quadruped(quad_model):
    om = oracle.OracleModel(quad_model.dump())
    qpos, qvel = mjb200.models.quadruped_initial_state(24)
    ob = oracle.OracleBatch(om, 24)
    ob.set_state(qpos, qvel)
    checked = 0
    for s in range(40):
        ob.set_ctrl(mjb200.models.quadruped_controls(24, s // 4))
        ob.step(1, nthread=4)
        if s % 10 == 9:
            for env in ob.envs:
                assert env.d.status == 0
                types = env.efc()["type"]
                # condim 3 pyramidal: 4 rows per contact
                assert (types == 2).sum() == 4 * env.d.ncon
                assert set(types.tolist()) <= {1, 2}
                res, f, force = _gauss_residual(om, env)
                assert res < 1e-6
                np.testing.assert_allclose(force, f, atol=1e-6 * max(1.0, np.abs(f).max(initial=0.0)))
                checked += 1
    assert checked == 96


def test_quadruped_mass_matrix_spd(quad_model):
    om = oracle.OracleModel(quad_model.dump())
    qpos, qvel = mjb200.models.quadruped_initial_state(8)
    for e in range(8):
        env = oracle.OracleEnv(om)
        env.a["qpos"][:] = qpos[e]
        env.a["qvel"][:] = qvel[e]
        env.step()
        M = env.a["M"].reshape(om.nv, om.nv)
        np.testing.assert_allclose(M, M.T, atol=1e-12)
        assert np.linalg.eigvalsh(M).min() > 0


def test_batch_threads_deterministic(quad_model):
    om = oracle.OracleModel(quad_model.dump())
    qpos, qvel = mjb200.models.quadruped_initial_state(16)
    out = []
    for nthread in (1, 4):
        ob = oracle.OracleBatch(om, 16)
        ob.set_state(qpos, qvel)
        ob.set_ctrl(mjb200.models.quadruped_controls(16, 0))
        ob.step(8, nthread=nthread)
        out.append(ob.state())
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("condim,rows", [(1, 1), (3, 4), (4, 6), (6, 10)])
def test_rows_per_contact_by_condim(condim, rows):
    """The reference's legacy structural rule (tests/test_friction_condim3.cpp,
    tests/test_friction_condim46.cpp): pyramidal contacts give 2 (condim - 1)
    rows, frictionless contacts 1."""
    xml = wrap(PLANE.replace('size="5 5 0.1"', f'size="5 5 0.1" condim="{condim}"') +
               f'<body pos="0 0 0.049"><freejoint/><geom type="box" size="0.2 0.1 0.05" mass="1" condim="{condim}"/></body>')
    om, env = env_from_xml(xml)
    env.step()
    assert env.d.ncon == 4
    assert env.d.nefc == 4 * rows
    res, f, force = _gauss_residual(om, env)
    assert res < 1e-6


def test_ray_known_answers():
    """Closed-form ray hits: plane from above only, sphere, box from outside
    and inside, capsule cap, cylinder disc, body exclusion."""
    xml = wrap(PLANE + '<body pos="0 0 1"><freejoint/><geom type="sphere" size="0.2"/></body>'
                       '<body pos="2 0 1"><geom type="box" size="0.1 0.2 0.3"/></body>'
                       '<body pos="0 2 1"><geom type="capsule" size="0.1 0.3"/></body>'
                       '<body pos="0 -2 1"><geom type="cylinder" size="0.1 0.3"/></body>')
    om, env = env_from_xml(xml)
    env.kinematics()
    inc = np.ones(om.ngeom, np.int32)
    t, g = env.ray([0, 0, 3], [0, 0, -1], inc)
    assert (t, g) == (pytest.approx(1.8), 1)                 # sphere top at z = 1.2
    t, g = env.ray([5, 5, 1], [0, 0, -2], inc)
    assert (t, g) == (pytest.approx(0.5), 0)                 # plane, t in units of vec
    assert env.ray([5, 5, -1], [0, 0, 1], inc) == (-1, -1)   # plane not hit from below
    t, g = env.ray([2, 0, 1], [1, 0, 0], inc)
    assert (t, g) == (pytest.approx(0.1), 2)                 # box exit from inside
    t, g = env.ray([0, 2, 3], [0, 0, -1], inc)
    assert (t, g) == (pytest.approx(3 - 1.4), 3)             # capsule cap top at z = 1.4
    t, g = env.ray([0, -2, 3], [0, 0, -1], inc)
    assert (t, g) == (pytest.approx(3 - 1.3), 4)             # cylinder disc at z = 1.3
    inc[1] = 0
    t, g = env.ray([0, 0, 3], [0, 0, -1], inc)
    assert g == 0 and t == pytest.approx(3.0)               # sphere excluded: the plane


def test_box_box_face_contact():
    """A 0.2 x 0.1 x 0.1 (half sizes) box sunk 1 mm into a larger static box:
    4 contacts at the small box's bottom corners, normal +z (geom 1 -> 2)."""
    xml = wrap('<geom type="box" size="0.5 0.5 0.1" pos="0 0 0.1"/>'
               '<body pos="0.05 -0.03 0.299"><freejoint/><geom type="box" size="0.2 0.1 0.1" mass="1"/></body>')
    om, env = env_from_xml(xml)
    env.step()
    cons = env.contacts()
    assert env.d.ncon == 4
    for c in cons:
        assert c[12] == pytest.approx(-0.001, abs=1e-9)
        np.testing.assert_allclose(c[3:6], [0, 0, 1], atol=1e-12)
        assert c[2] == pytest.approx(0.2 - 0.0005, abs=1e-9)
    xy = sorted((round(c[0], 9), round(c[1], 9)) for c in cons)
    assert xy == sorted([(round(0.05 + sx * 0.2, 9), round(-0.03 + sy * 0.1, 9)) for sx in (-1, 1) for sy in (-1, 1)])
    assert env.d.nefc == 16


def test_box_box_edge_contact_and_separation():
    """Two boxes whose edges cross (rotated 45 deg about x and about y): one
    edge-edge contact on the line between the centres; far apart: none."""
    c, s = np.cos(np.pi / 8), np.sin(np.pi / 8)
    h = 0.1 * np.sqrt(2)
    gap = -0.002
    xml = wrap(f'<geom type="box" size="0.1 0.1 0.1" quat="{c} {s} 0 0" pos="0 0 0"/>'
               f'<body pos="0 0 {2 * h + gap}" quat="{c} 0 {s} 0"><freejoint/><geom type="box" size="0.1 0.1 0.1" mass="1"/></body>',
               option='<option timestep="0.005" gravity="0 0 0"/>')
    om, env = env_from_xml(xml)
    env.step()
    assert env.d.ncon == 1
    con = env.contacts()[0]
    assert con[12] == pytest.approx(gap, abs=1e-9)
    np.testing.assert_allclose(con[3:6], [0, 0, 1], atol=1e-9)
    np.testing.assert_allclose(con[0:3], [0, 0, h + gap / 2], atol=1e-9)
    xml_far = xml.replace(f'pos="0 0 {2 * h + gap}"', 'pos="0 0 1"')
    om, env = env_from_xml(xml_far)
    env.step()
    assert env.d.ncon == 0


def test_box_stack_comes_to_rest():
    m_ = 1.5
    xml = wrap(PLANE + '<body pos="0 0 0.1"><freejoint/><geom type="box" size="0.3 0.3 0.1" mass="4"/></body>'
                       f'<body pos="0.02 0.01 0.3"><freejoint/><geom type="box" size="0.15 0.1 0.1" mass="{m_}"/></body>')
    om, env = env_from_xml(xml)
    for _ in range(800):
        env.step()
    assert env.d.status == 0
    assert abs(env.a["qvel"]).max() < 1e-4
    types = env.efc()["type"]
    # 4 floor contacts + 4 box-box contacts, all pyramidal
    assert env.d.ncon == 8 and (types == 2).sum() == 32
    cons = env.contacts()
    bb = [i for i in range(8) if int(cons[i][14]) == 1 and int(cons[i][15]) == 2]
    assert len(bb) == 4
    rows = env.efc()["force"].reshape(-1, 4)
    assert rows[bb].sum() == pytest.approx(m_ * G, rel=1e-3)


def test_joint_equality_couples_joints():
    """Joint equality q_b - q_b0 = 0.5 (q_a - q_a0): one bilateral row ahead
    of every other row, Gauss-optimal solutions, and the coupling held to
    within the soft constraint's tracking error while the pendulum swings."""
    xml = wrap('<body><joint name="a" type="hinge" axis="0 1 0" damping="0.2" frictionloss="0.01"/>'
               '<geom type="capsule" fromto="0 0 0 0 0 -0.3" size="0.02" mass="1"/>'
               '<body pos="0 0 -0.3"><joint name="b" type="hinge" axis="0 1 0" damping="0.2"/>'
               '<geom type="capsule" fromto="0 0 0 0 0 -0.3" size="0.02" mass="1"/></body></body>',
               extra="") .replace("</mujoco>", '<equality><joint joint1="b" joint2="a" polycoef="0 0.5 0 0 0"/></equality></mujoco>')
    om, env = env_from_xml(xml)
    env.a["qpos"][:] = [0.8, -0.3]
    env.step()
    t = env.efc()["type"]
    assert list(t[:2]) == [5, 0]                     # equality row first, then frictionloss
    res, f, force = _gauss_residual(om, env)
    assert res < 1e-6
    np.testing.assert_allclose(force[:1], f[:1], rtol=1e-9)
    worst = 0.0
    for i in range(1500):
        env.step()
        q = env.a["qpos"]
        if i > 100:
            worst = max(worst, abs(q[1] - 0.5 * q[0]))
    assert worst < 0.02                              # soft-constraint tracking error while swinging
    assert abs(env.a["qpos"][0]) > 1e-3              # it did swing


def _tendon_chain():
    m = mjb200.load_model_from_string(mjb200.models.tendon_chain_xml(8))
    om = oracle.OracleModel(m.dump())
    return m, om


# tendon wraps of the tendon chain: tendon -> {dof: coef}
_TENDON_J = [{0: 1.0, 1: 0.5}, {2: 1.0, 3: -1.0, 4: 0.5}, {1: 1.0, 5: 1.0}, {6: 1.0, 7: 0.7}, {4: 1.0, 5: -0.3}]


def _tjac(t, nv=8):
    J = np.zeros(nv)
    for k, c in _TENDON_J[t].items():
        J[k] = c
    return J


def test_tendon_compile_known_answers():
    """Fixed tendons compile to their wraps; auto limits from range=; rest
    length and invweight J M^-1 J^T at qpos0; springlength defaults to the
    rest length; tendon equality invweight = sum of both tendons'."""
    m, om = _tendon_chain()
    d = m.dump()
    assert list(d["tendon_num"]) == [2, 3, 2, 2, 2]
    assert list(d["tendon_limited"]) == [1, 1, 0, 0, 0]
    np.testing.assert_allclose(d["tendon_lengthspring"].reshape(-1, 2)[0], [-0.05, 0.05])
    np.testing.assert_allclose(d["tendon_lengthspring"].reshape(-1, 2)[2], [0.0, 0.0])
    assert list(d["actuator_trntype"]) == [3, 3] and list(d["actuator_trnid"]) == [0, 1]
    env = oracle.OracleEnv(om)
    env.step()  # at qpos0: M is the mass matrix there
    M = env.a["M"].reshape(8, 8)
    for t in range(5):
        J = _tjac(t)
        assert d["tendon_invweight0"][t] == pytest.approx(J @ np.linalg.solve(M, J), rel=1e-9)
    assert d["eq_invweight"][0] == pytest.approx(d["tendon_invweight0"][3] + d["tendon_invweight0"][4], rel=1e-12)
    bad = mjb200.models.tendon_chain_xml(8).replace('<fixed name="t4">', '<spatial name="t5"><pulley divisor="2"/></spatial><fixed name="t4">')
    with pytest.raises(Exception, match="pulley must follow a site"):
        mjb200.load_model_from_string(bad)


def test_tendon_passive_actuator_and_rows():
    """Passive force J^T (spring with dead band - damping * velocity), tendon
    actuator force gear * force * J, and the row order equality -> tendon
    frictionloss -> tendon limits, each row's J, aref and the Gauss
    optimality of the solution."""
    m, om = _tendon_chain()
    env = oracle.OracleEnv(om)
    q = np.array([0.5, 0.2, 0.3, -0.2, 0.1, -0.1, 0.2, 0.1])   # t0 = 0.6 > 0.3, t1 = 0.55 > 0.4
    v = np.array([0.3, -0.2, 0.1, 0.4, -0.3, 0.2, 0.1, -0.1])
    env.a["qpos"][:] = q
    env.a["qvel"][:] = v
    env.a["ctrl"][:2] = [0.7, 0.1]
    env.step()
    L = [_tjac(t) @ q for t in range(5)]
    V = [_tjac(t) @ v for t in range(5)]
    # passive: dof damping 0.02, t0 spring k=2 dead band [-0.05, 0.05] + damper 0.05, t2 spring k=1 to rest 0
    f0 = 2.0 * (0.05 - L[0]) - 0.05 * V[0]
    f2 = 1.0 * (0.0 - L[2])
    pas = -0.02 * v + _tjac(0) * f0 + _tjac(2) * f2
    np.testing.assert_allclose(env.a["qfrc_passive"], pas, rtol=1e-12, atol=1e-14)
    # actuators: motor on t0 (ctrl 0.7), position kp 5 on t1 (target 0.1)
    act = _tjac(0) * 0.7 + _tjac(1) * 5.0 * (0.1 - L[1])
    np.testing.assert_allclose(env.a["qfrc_actuator"], act, rtol=1e-12, atol=1e-14)
    e = env.efc()
    assert list(e["type"]) == [5, 0, 0, 1, 1]
    np.testing.assert_allclose(e["J"][0], _tjac(3) - 0.8 * _tjac(4), atol=1e-15)
    np.testing.assert_allclose(e["J"][1], _tjac(0))
    np.testing.assert_allclose(e["J"][2], _tjac(2))
    np.testing.assert_allclose(e["J"][3], -_tjac(0))     # upper side of t0
    np.testing.assert_allclose(e["J"][4], -_tjac(1))     # upper side of t1
    # aref of the limit row: -b (J v) - k imp pos with pos = 0.3 - t0 (< 0, saturated imp = dmax)
    dmax, tc = 0.95, 0.02
    k, b = 1 / (dmax ** 2 * tc ** 2), 2 / (dmax * tc)
    assert e["aref"][3] == pytest.approx(-b * (-V[0]) - k * dmax * (0.3 - L[0]), rel=1e-12)
    res, f, force = _gauss_residual(om, env)
    assert res < 1e-6


def test_tendon_limit_and_equality_hold_in_rollout():
    """Rolled out under random tendon controls, t0 stays near [-0.3, 0.3]
    (soft limit), the equality t3 = 0.8 t4 holds to the soft-constraint
    tracking error, and no env is flagged."""
    m, om = _tendon_chain()
    env = oracle.OracleEnv(om)
    g = np.random.default_rng(2)
    env.a["qpos"][:] = g.normal(0, 0.1, 8)
    worst_lim, worst_eq = 0.0, 0.0
    for s in range(1500):
        if s % 100 == 0:
            env.a["ctrl"][:2] = [g.uniform(-1, 1), g.uniform(-0.4, 0.4)]
        env.step()
        assert env.d.status == 0
        q = env.a["qpos"]
        if s > 50:
            worst_lim = max(worst_lim, abs(_tjac(0) @ q) - 0.3)
            worst_eq = max(worst_eq, abs(_tjac(3) @ q - 0.8 * (_tjac(4) @ q)))
    assert worst_lim < 0.05 and worst_eq < 0.05


def _quat2mat(q):
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


_FLOATER = ('<mujoco><option timestep="0.005" gravity="0 0 -9.81" magnetic="0.2 -0.5 0.1"/><worldbody>'
            '<body name="b" pos="0 0 1"><freejoint/><geom type="box" size="0.1 0.2 0.3" mass="2"/>'
            '<site name="s" pos="0.1 -0.05 0.2"/></body></worldbody>'
            '<sensor><gyro site="s"/><velocimeter site="s"/><accelerometer site="s"/><magnetometer site="s"/>'
            '<framequat objtype="site" objname="s"/><framexaxis objtype="site" objname="s"/><framezaxis objtype="site" objname="s"/>'
            '<framepos objtype="xbody" objname="b"/><touch site="s"/></sensor></mujoco>')


def test_sensor_known_answers_free_body():
    """Free body with a site at p (identity site frame), start state q0, v0:
    gyro = the free joint's local angular velocity, velocimeter = R^T v +
    w_local x p, magnetometer = R^T magnetic, frame axes = columns of R,
    framequat = +-q0 with w >= 0, framepos(xbody) = root position; the
    accelerometer reads R^T(-g) without history and, for a non-rotating
    body in free fall, 0 once the previous velocity is known; touch (outside
    the batched set) reads 0."""
    m = mjb200.load_model_from_string(_FLOATER)
    om = oracle.OracleModel(m.dump())
    env = oracle.OracleEnv(om)
    q0 = np.array([0.3, -0.2, 1.1, 0.6, 0.3, -0.5, 0.2])
    q0[3:] /= np.linalg.norm(q0[3:])
    v0 = np.array([0.4, -0.3, 0.2, 1.5, -0.7, 0.9])
    env.a["qpos"][:] = q0
    env.a["qvel"][:] = v0
    sd = env.step_sensors()
    R = _quat2mat(q0[3:])
    p = np.array([0.1, -0.05, 0.2])
    wl = v0[3:]
    np.testing.assert_allclose(sd[0:3], wl, atol=1e-12)
    np.testing.assert_allclose(sd[3:6], R.T @ v0[:3] + np.cross(wl, p), atol=1e-12)
    np.testing.assert_allclose(sd[6:9], R.T @ np.array([0, 0, 9.81]), atol=1e-12)
    np.testing.assert_allclose(sd[9:12], R.T @ np.array([0.2, -0.5, 0.1]), atol=1e-12)
    qs = q0[3:] * (1 if q0[3] >= 0 else -1)
    np.testing.assert_allclose(sd[12:16], qs, atol=1e-12)
    np.testing.assert_allclose(sd[16:19], R[:, 0], atol=1e-12)
    np.testing.assert_allclose(sd[19:22], R[:, 2], atol=1e-12)
    np.testing.assert_allclose(sd[22:25], q0[:3], atol=1e-12)
    assert sd[25] == 0.0
    # no rotation: free fall, accelerometer 0 once a previous velocity exists
    env.a["qvel"][3:] = 0.0
    env.step_sensors()
    sd = env.step_sensors()
    np.testing.assert_allclose(sd[6:9], 0.0, atol=1e-9)
    env.reset_sensor_history()
    sd = env.step_sensors()
    R = _quat2mat(env.a["qpos"][3:])   # rotation unchanged (no angular velocity)
    np.testing.assert_allclose(sd[6:9], R.T @ np.array([0, 0, 9.81]), atol=1e-9)


def test_sensor_rig_joint_tendon_actuator_values():
    """Joint, ball, actuator (joint and tendon transmission), tendon and
    joint actuator force sensors equal the start state's values; sensor
    adr / dim follow the declaration order; the relative frame sensor and
    the touch sensor read 0."""
    m = mjb200.load_model_from_string(mjb200.models.sensor_xml())
    om = oracle.OracleModel(m.dump())
    S = {nm: (t, a, dm) for nm, t, a, dm in m.sensors()}
    assert S["imu_gyro"] == (3, 0, 3) and S["imu_acc"][1:] == (3, 3) and m.nsensordata == sum(v[2] for v in S.values())
    q, v = mjb200.models.sensor_state(m, 1, 5)
    env = oracle.OracleEnv(om)
    env.a["qpos"][:] = q[0]
    env.a["qvel"][:] = v[0]
    env.a["ctrl"][:4] = [0.3, -0.2, 0.05, 0.4]
    sd = env.step_sensors()
    d = m.dump()
    jq, jd = d["jnt_qposadr"], d["jnt_dofadr"]
    val = lambda nm: sd[S[nm][1]: S[nm][1] + S[nm][2]]
    # joints: 0 free, 1 shoulder, 2 elbow, 3 slide, 4 ball
    assert val("q_sh")[0] == q[0, jq[1]] and val("v_sh")[0] == v[0, jd[1]]
    assert val("q_sl")[0] == q[0, jq[3]] and val("v_sl")[0] == v[0, jd[3]]
    np.testing.assert_allclose(val("ball_q"), q[0, jq[4]: jq[4] + 4] / np.linalg.norm(q[0, jq[4]: jq[4] + 4]))
    np.testing.assert_allclose(val("ball_w"), v[0, jd[4]: jd[4] + 3])
    assert val("ap_sh")[0] == pytest.approx(2 * q[0, jq[1]]) and val("av_sh")[0] == pytest.approx(2 * v[0, jd[1]])
    tl = q[0, jq[1]] + 0.5 * q[0, jq[2]]
    tv = v[0, jd[1]] + 0.5 * v[0, jd[2]]
    assert val("t_pos")[0] == pytest.approx(tl) and val("t_vel")[0] == pytest.approx(tv)
    assert val("ap_t")[0] == pytest.approx(0.5 * tl) and val("av_t")[0] == pytest.approx(0.5 * tv)
    # shoulder: motor gear 2 (ctrl 0.3) + tendon motor gear 0.5 (ctrl 0.4) through J = 1
    assert val("f_sh")[0] == pytest.approx(2 * 0.3 + 0.5 * 0.4 * 1.0)
    # slide: position actuator kp 15, gear 1.5, target 0.05
    assert val("f_sl")[0] == pytest.approx(1.5 * 15 * (0.05 - 1.5 * q[0, jq[3]]))
    np.testing.assert_allclose(val("fore_xpos"), env.a["xpos"][3 * 3: 3 * 4])
    np.testing.assert_allclose(val("com"), env.a["subtree_com"][3:6])
    assert not val("touch_tip").any() and not val("rel_pos").any()


def _pair_contacts(g1, g2, pose1, pose2, margin=0.0):
    """Contacts of one geom pair (two free bodies, no gravity) at the given
    poses (pos3 + quat4 each), from the oracle's collision stage alone."""
    import ctypes as C
    xml = (f'<mujoco><option gravity="0 0 0"/><worldbody><body name="a"><freejoint/><geom {g1} margin="{margin}"/></body>'
           f'<body name="b" pos="0 0 1"><freejoint/><geom {g2} margin="{margin}"/></body></worldbody></mujoco>')
    m = mjb200.load_model_from_string(xml)
    om = oracle.OracleModel(m.dump())
    env = oracle.OracleEnv(om)
    env.a["qpos"][:] = np.concatenate([pose1, pose2])
    oracle.lib.oracle_kinematics(C.byref(om.c), C.byref(env.d))
    oracle.lib.oracle_collide(C.byref(om.c), C.byref(env.d))
    return env.contacts(), env.d.status, m.dump()["geom_type"]


def _rand_quat(g):
    q = g.normal(size=4)
    return q / np.linalg.norm(q)


def test_convex_gjk_epa_curved_known_answers():
    """GJK distance (separated, within margin) and EPA + Newton refinement
    (penetrating) between a sphere and a sphere-shaped ellipsoid, and
    between two sphere-shaped ellipsoids, against the closed form: dist =
    |c2 - c1| - r1 - r2, normal along c2 - c1, position at the midpoint of
    the surface points."""
    g = np.random.default_rng(7)
    for g1, r1, g2, r2 in (('type="sphere" size="0.1"', 0.1, 'type="ellipsoid" size="0.2 0.2 0.2"', 0.2),
                           ('type="ellipsoid" size="0.15 0.15 0.15"', 0.15, 'type="ellipsoid" size="0.2 0.2 0.2"', 0.2)):
        for dist in (0.1, 0.01, -0.02, -0.12):
            u = g.normal(size=3)
            u /= np.linalg.norm(u)
            c1 = g.normal(size=3) * 0.3
            c2 = c1 + u * (r1 + r2 + dist)
            cs, st, gt = _pair_contacts(g1, g2, np.r_[c1, _rand_quat(g)], np.r_[c2, _rand_quat(g)], margin=0.2)
            assert st == 0 and len(cs) == 1
            sgn = 1 if gt[0] <= gt[1] else -1   # pair order is by geom type
            assert cs[0, 12] == pytest.approx(dist, abs=1e-8)
            np.testing.assert_allclose(cs[0, 3:6], sgn * u, atol=1e-6)
            mid = 0.5 * ((c1 + r1 * u) + (c2 - r2 * u))
            np.testing.assert_allclose(cs[0, :3], mid, atol=1e-6)


def test_convex_capsule_side_against_curved_known_answer():
    """Capsule side (its core segment is flat along the axis, so the depth
    has a kink there and curvature across it) against a sphere-shaped
    ellipsoid: dist = distance from the centre to the core segment - r - R,
    normal from the closest segment point to the centre."""
    g = np.random.default_rng(11)
    r, hl, R = 0.03, 0.06, 0.05
    for dist in (0.02, -0.004, -0.03):
        for trial in range(4):
            q1 = _rand_quat(g)
            w, x, y, z = q1
            axis = np.array([2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)])
            perp = np.cross(axis, g.normal(size=3))
            perp /= np.linalg.norm(perp)
            s = g.uniform(-0.8, 0.8) * hl
            c1 = g.normal(size=3) * 0.1
            c2 = c1 + s * axis + perp * (r + R + dist)
            cs, st, gt = _pair_contacts('type="capsule" size="%g %g"' % (r, hl), 'type="ellipsoid" size="%g %g %g"' % (R, R, R),
                                        np.r_[c1, q1], np.r_[c2, _rand_quat(g)], margin=0.05)
            assert len(cs) == 1
            assert cs[0, 12] == pytest.approx(dist, abs=1e-8)
            np.testing.assert_allclose(cs[0, 3:6], perp, atol=1e-6)   # capsule (3) is geom1


def test_convex_mesh_cube_matches_box_colliders():
    """A mesh whose hull is a 0.2 m cube against a sphere and a capsule:
    GJK / EPA on the hull give the analytic sphere-box depth and normal
    (face, edge and vertex regions, separated and penetrating) and the
    capsule-box distance when separated; when a capsule penetrates, the
    minimum translation distance is at least the deepest-point depth of the
    analytic capsule-box collider."""
    cube = " ".join(f"{x} {y} {z}" for x in (-0.1, 0.1) for y in (-0.1, 0.1) for z in (-0.1, 0.1))
    g = np.random.default_rng(8)
    for other in ('type="sphere" size="0.07"', 'type="capsule" size="0.04 0.08"'):
        for trial in range(12):
            q1, q2 = _rand_quat(g), _rand_quat(g)
            c2 = g.uniform(-0.22, 0.22, size=3)
            xml_mesh = f'type="mesh" mesh="cube"'
            mesh_model = ('<asset><mesh name="cube" vertex="' + cube + '"/></asset>')
            import ctypes as C
            outs = []
            for shape in (xml_mesh, 'type="box" size="0.1 0.1 0.1"'):
                xml = (f'<mujoco><option gravity="0 0 0"/>{mesh_model}<worldbody><body name="a"><freejoint/><geom {shape} margin="0.1"/></body>'
                       f'<body name="b" pos="0 0 1"><freejoint/><geom {other} margin="0.1"/></body></worldbody></mujoco>')
                m = mjb200.load_model_from_string(xml)
                om = oracle.OracleModel(m.dump())
                env = oracle.OracleEnv(om)
                env.a["qpos"][:] = np.concatenate([[0, 0, 0], q1, c2, q2])
                oracle.lib.oracle_kinematics(C.byref(om.c), C.byref(env.d))
                oracle.lib.oracle_collide(C.byref(om.c), C.byref(env.d))
                outs.append((env.contacts(), m.dump()["geom_type"]))
            (cm, tm), (cb, tb) = outs
            assert len(cm) == len(cb)
            if len(cm):
                # mesh (type 7) and box (6) are both geom2 of their pair
                if other.startswith('type="sphere"') or cb[0, 12] > 0:
                    assert cm[0, 12] == pytest.approx(cb[0, 12], abs=1e-7)
                    np.testing.assert_allclose(cm[0, 3:6], cb[0, 3:6], atol=1e-5)
                else:
                    assert cm[0, 12] <= cb[0, 12] + 1e-9


def test_convex_flat_and_order_symmetry():
    """Cylinder standing on a box: depth and normal exact, position between
    the faces; swapping the two bodies flips nothing in dist and keeps the
    normal pointing from geom1 to geom2."""
    I = [1, 0, 0, 0]
    cs, st, gt = _pair_contacts('type="box" size="0.3 0.3 0.1"', 'type="cylinder" size="0.1 0.2"', np.r_[0, 0, 0, I], np.r_[0.05, 0.02, 0.29, I])
    assert len(cs) == 1 and cs[0, 12] == pytest.approx(-0.01, abs=1e-9)
    np.testing.assert_allclose(cs[0, 3:6], [0, 0, -1], atol=1e-9)   # cylinder (type 5) is geom1
    assert cs[0, 2] == pytest.approx(0.095, abs=1e-9)
    g = np.random.default_rng(9)
    for trial in range(8):
        p1 = np.r_[g.normal(size=3) * 0.1, _rand_quat(g)]
        p2 = np.r_[p1[:3] + g.normal(size=3) * 0.12, _rand_quat(g)]
        a, _, ta = _pair_contacts('type="ellipsoid" size="0.12 0.08 0.05"', 'type="cylinder" size="0.05 0.07"', p1, p2, margin=0.05)
        b, _, tb = _pair_contacts('type="cylinder" size="0.05 0.07"', 'type="ellipsoid" size="0.12 0.08 0.05"', p2, p1, margin=0.05)
        assert len(a) == len(b)
        if len(a):
            assert a[0, 12] == pytest.approx(b[0, 12], abs=1e-7)
            np.testing.assert_allclose(a[0, 3:6], b[0, 3:6], atol=1e-5)


def _dp(a):
    import ctypes as C
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(C.POINTER(C.c_double))


_CHAIN3 = ('<mujoco><option timestep="0.002"/><worldbody>'
           '<body><joint type="hinge" axis="0 1 0"/><geom type="capsule" fromto="0 0 0 0.3 0 0" size="0.03" mass="1"/>'
           '<body pos="0.3 0 0"><joint type="hinge" axis="1 0 0"/><geom type="capsule" fromto="0 0 0 0.25 0 0.1" size="0.03" mass="0.6"/>'
           '<body pos="0.25 0 0.1"><joint type="hinge" axis="0 1 0"/><geom type="sphere" size="0.05" mass="0.4" pos="0.1 0 0"/>'
           '</body></body></body></worldbody></mujoco>')


def test_gravcomp_known_answers():
    """Gravity compensation (gravcomp = 1 on every body) cancels gravity: at
    zero velocity qacc = 0; gravcomp = 0.5 halves the zero-velocity
    acceleration of the uncompensated chain."""
    q = np.array([0.3, -0.4, 0.7])
    acc = {}
    for gc in ("0", "0.5", "1"):
        xml = _CHAIN3.replace("<body>", f'<body gravcomp="{gc}">').replace('<body pos', f'<body gravcomp="{gc}" pos')
        om, env = env_from_xml(xml)
        env.a["qpos"][:] = q
        env.step()
        acc[gc] = env.a["qacc"].copy()
    np.testing.assert_allclose(acc["1"], 0.0, atol=1e-12)
    np.testing.assert_allclose(acc["0.5"], 0.5 * acc["0"], rtol=1e-10)
    assert np.abs(acc["0"]).max() > 1.0


def test_com_offset_and_drag_known_answers():
    """Per-env COM offset: a hinged sphere (COM at L on the arm, axis y,
    horizontal arm) accelerates at m g (L + d) / (I + m (L + d)^2) with the
    COM moved by d along the arm.  Per-env drag: a free body in zero gravity
    (COM at its origin) decelerates at -k |v| v / m."""
    import ctypes as C
    L, mass, r = 0.3, 2.0, 0.05
    xml = (f'<mujoco><option timestep="0.002"/><worldbody><body><joint type="hinge" axis="0 1 0"/>'
           f'<geom type="sphere" size="{r}" pos="{L} 0 0" mass="{mass}"/></body></worldbody></mujoco>')
    om, env = env_from_xml(xml)
    I = 0.4 * mass * r * r
    for d in (0.0, 0.05, -0.1):
        env.a["qpos"][:] = 0
        env.a["qvel"][:] = 0
        cd = np.zeros((2, 3))
        cd[1, 0] = d
        keep = np.ascontiguousarray(cd.reshape(-1))
        rand = oracle.ORand(None, 1.0, None, keep.ctypes.data_as(C.POINTER(C.c_double)), None)
        env.step(0, rand)
        Ld = L + d
        assert env.a["qacc"][0] == pytest.approx(mass * 9.81 * Ld / (I + mass * Ld * Ld), rel=1e-10)
    xml = ('<mujoco><option timestep="0.002" gravity="0 0 0"/><worldbody><body><freejoint/>'
           '<geom type="box" size="0.1 0.2 0.3" mass="3"/></body></worldbody></mujoco>')
    om, env = env_from_xml(xml)
    v = np.array([0.4, -1.2, 0.7])
    env.a["qvel"][:3] = v
    k = np.array([0.8])
    rand = oracle.ORand(None, 1.0, None, None, k.ctypes.data_as(C.POINTER(C.c_double)))
    env.step(0, rand)
    np.testing.assert_allclose(env.a["qacc"][:3], -0.8 * np.linalg.norm(v) * v / 3.0, rtol=1e-10)
    np.testing.assert_allclose(env.a["qacc"][3:], 0.0, atol=1e-12)


def test_spatial_tendon_wrap_known_answers():
    """Static sites around a world sphere / cylinder: the wrapped length is
    2 sqrt(a^2 - r^2) + r (pi - 2 acos(r / a)) for points at +-a through the
    centre; a cylinder adds the axial rise as a helix, sqrt(L^2 + dz^2); a
    path that misses the geom is straight; a pulley divides the next branch."""
    a, r, dz = 0.3, 0.1, 0.2
    L2 = 2 * np.sqrt(a * a - r * r) + r * (np.pi - 2 * np.arccos(r / a))
    xml = (f'<mujoco><worldbody><geom name="ball" type="sphere" size="{r}" contype="0" conaffinity="0"/>'
           f'<geom name="can" type="cylinder" size="{r} 0.5" pos="0 2 0" contype="0" conaffinity="0"/>'
           f'<site name="s0" pos="{-a} 0 0"/><site name="s1" pos="{a} 0 0"/><site name="s2" pos="{a} 0.5 0.4"/>'
           f'<site name="c0" pos="{-a} 2 0"/><site name="c1" pos="{a} 2 {dz}"/><site name="up" pos="0 0 1"/>'
           '<body><joint type="slide" axis="0 0 1"/><geom type="sphere" size="0.01" mass="1" contype="0" conaffinity="0"/></body></worldbody>'
           '<tendon><spatial><site site="s0"/><geom geom="ball"/><site site="s1"/></spatial>'
           '<spatial><site site="c0"/><geom geom="can"/><site site="c1"/></spatial>'
           '<spatial><site site="s0"/><geom geom="ball" sidesite="up"/><site site="s2"/></spatial>'
           '<spatial><site site="s0"/><site site="s1"/><pulley divisor="4"/><site site="s1"/><site site="s2"/></spatial>'
           '</tendon></mujoco>')
    om, env = env_from_xml(xml)
    l0 = env.tendon(0)[0]
    assert l0 == pytest.approx(L2, rel=1e-12)
    assert env.tendon(1)[0] == pytest.approx(np.sqrt(L2 * L2 + dz * dz), rel=1e-12)
    # s0 -> s2 with the side site above: the straight line misses the ball (it
    # passes above the centre, on the side site's side) -> straight
    s0, s2 = np.array([-a, 0, 0]), np.array([a, 0.5, 0.4])
    t = (np.dot(-s0, s2 - s0) / np.dot(s2 - s0, s2 - s0))
    assert np.linalg.norm(s0 + t * (s2 - s0)) > r
    assert env.tendon(2)[0] == pytest.approx(np.linalg.norm(s2 - s0), rel=1e-12)
    assert env.tendon(3)[0] == pytest.approx(2 * a + np.linalg.norm(s2 - np.array([a, 0, 0])) / 4, rel=1e-12)


def test_spatial_tendon_jacobian_matches_finite_differences():
    """On the wrapped arm, the oracle's tendon Jacobian equals the finite
    difference of its length (tangent points moving with their geom: the
    envelope of the shortest wrapped path)."""
    m = mjb200.load_model_from_string(mjb200.models.spatial_tendon_xml())
    om = oracle.OracleModel(m.dump())
    env = oracle.OracleEnv(om)
    g = np.random.default_rng(3)
    for trial in range(6):
        q = np.array([g.uniform(-0.8, 0.8), g.uniform(-1.5, 1.5), g.uniform(-0.1, 0.1)])
        for t in range(3):
            env.a["qpos"][:] = q
            _, _, J = env.tendon(t)
            fd = np.zeros(3)
            for i in range(3):
                for sg in (1, -1):
                    qq = q.copy()
                    qq[i] += sg * 1e-6
                    env.a["qpos"][:] = qq
                    fd[i] += sg * env.tendon(t)[0] / 2e-6
            np.testing.assert_allclose(J, fd, atol=1e-7)


def _cone_force(D0, mu, fric, y):
    """MuJoCo's elliptic cone in numpy, written from the cost rather than
    shared with the C code: s(y) over one contact's rows with U = (mu y0,
    fric_j y_j), N = U0, T = |U_t|; top zone (N >= mu T) zero, bottom zone
    (mu N + T <= 0) quadratic in every row, middle 0.5 Dm (N - mu T)^2 with
    Dm = D0 / (mu^2 (1 + mu^2)).  Returns (cost, force = -ds/dy)."""
    U = np.concatenate([[mu * y[0]], fric * y[1:]])
    N, T = U[0], np.linalg.norm(U[1:])
    if N >= mu * T or (T <= 0 and N >= 0):
        return 0.0, np.zeros_like(y)
    if mu * N + T <= 0 or (T <= 0 and N < 0):
        return None, None   # bottom: the caller handles it with per-row D
    Dm = D0 / (mu * mu * (1 + mu * mu))
    g = np.concatenate([[mu], -mu * U[1:] / T * fric])   # d(N - mu T)/dy
    return 0.5 * Dm * (N - mu * T) ** 2, -Dm * (N - mu * T) * g


def _elliptic_cost_and_force(e, floss, y):
    cost, f, r = 0.0, np.zeros_like(y), 0
    while r < len(y):
        t = e["type"][r]
        if t == 4:
            dim = 1
            while r + dim < len(y) and e["type"][r + dim] == 6:
                dim += 1
            c, fc = _cone_force(e["D"][r], floss[r], floss[r + 1: r + dim], y[r: r + dim])
            if c is None:
                fc = -e["D"][r: r + dim] * y[r: r + dim]
                c = 0.5 * float(e["D"][r: r + dim] @ (y[r: r + dim] ** 2))
            cost += c
            f[r: r + dim] = fc
            r += dim
        else:
            assert t in (1, 3, 5)
            fr = -e["D"][r] * (y[r] if t == 5 else min(y[r], 0.0))
            cost += 0.5 * e["D"][r] * (y[r] ** 2 if t == 5 else min(y[r], 0.0) ** 2)
            f[r] = fr
            r += 1
    return cost, f


def _elliptic_box(condim, mu=0.5, impratio=1.0):
    om, env = env_from_xml(mjb200.models.pushed_box_xml("elliptic", condim, mu, impratio))
    env.a["qpos"][:] = 0
    env.a["qpos"][2] = -0.0005
    env.a["qpos"][3] = 1
    return om, env


@pytest.mark.parametrize("condim", [3, 4, 6])
@pytest.mark.parametrize("impratio", [1.0, 4.0])
def test_elliptic_cone_rows_and_gauss_optimality(condim, impratio):
    """Elliptic contacts: dim rows per contact (normal type 4, friction type
    6); R_j = R_n (mu_0 / mu_j)^2 / impratio; the Newton solution minimises
    the Gauss cost with the cone term (gradient residual ~0 and no random
    perturbation lowers the cost), for a box pushed with a tangential motor
    both below and above mu m g, at rest and sliding."""
    checked = 0
    for push in (1.0, 9.0):
        om, env = _elliptic_box(condim, impratio=impratio)
        for t in range(60):
            env.a["ctrl"][0] = push
            env.a["qvel"][1] = 0.05   # a sideways component: both tangents carry force
            env.step()
            assert env.d.status == 0
            e = env.efc()
            n = env.d.nefc
            nc = env.d.ncon
            if t % 3 or nc == 0:
                continue
            checked += 1
            assert n == nc * condim
            assert list(e["type"][:condim]) == [4] + [6] * (condim - 1)
            floss = env.a["efc_floss"][:n]
            R = 1 / e["D"]
            fr = np.array([0.5, 0.5, 0.02, 0.002, 0.002])
            for c in range(nc):
                r0 = c * condim
                assert floss[r0] == pytest.approx(0.5 / np.sqrt(impratio), rel=1e-12)
                for j in range(1, condim):
                    assert floss[r0 + j] == pytest.approx(fr[j - 1], rel=1e-12)
                    assert R[r0 + j] == pytest.approx(R[r0] * (0.5 / fr[j - 1]) ** 2 / impratio, rel=1e-9)
            nv = om.nv
            M = env.a["M"].reshape(nv, nv)
            qacc, qs = env.a["qacc"].copy(), env.a["qacc_smooth"]
            y = e["J"] @ qacc - e["aref"]

            def total(x):
                yx = e["J"] @ x - e["aref"]
                return 0.5 * (x - qs) @ M @ (x - qs) + _elliptic_cost_and_force(e, floss, yx)[0]

            c0, f = _elliptic_cost_and_force(e, floss, y)
            np.testing.assert_allclose(f, e["force"], atol=1e-8 * max(1.0, np.abs(f).max()))
            res = np.linalg.norm(M @ (qacc - qs) - e["J"].T @ f) / max(np.linalg.norm(M @ qs), 1.0)
            assert res < 1e-7, res
            # friction forces stay in the cone: |f_j / mu_j| over the tangents <= f_n / mu
            for c in range(nc):
                r0 = c * condim
                ft = f[r0 + 1: r0 + condim] / floss[r0 + 1: r0 + condim]
                assert f[r0] >= -1e-12
                assert np.linalg.norm(ft) <= f[r0] / floss[r0] * (1 + 1e-9) + 1e-12
            g = np.random.default_rng(condim)
            base = total(qacc)
            for k in range(20):
                d = g.normal(size=nv) * 10.0 ** g.uniform(-6, -2)
                assert total(qacc + d) >= base - 1e-10 * max(1.0, abs(base))
    assert checked >= 20


def test_elliptic_cone_stick_and_slide_known_answers():
    """Pushed box (m = 1 kg, mu = 0.5, condim 3): below mu m g it sticks
    (tangential velocity stays ~0); above it slides with a friction force on
    the cone boundary, |f_t| = mu f_n per contact, so the net tangential
    force is push - mu sum(f_n)."""
    om, env = _elliptic_box(3)
    for t in range(200):
        env.a["ctrl"][0] = 3.0
        env.step()
    assert abs(env.a["qvel"][0]) < 2e-3
    om, env = _elliptic_box(3)
    for t in range(200):
        env.a["ctrl"][0] = 9.0
        env.step()
        e = env.efc()
        if env.d.nefc == 0 or env.a["qvel"][0] < 0.05:
            continue
        f = e["force"].reshape(-1, 3)
        # every contact in the middle zone: friction on the boundary
        np.testing.assert_allclose(np.linalg.norm(f[:, 1:], axis=1), 0.5 * f[:, 0], rtol=1e-6)
    assert env.a["qvel"][0] > 0.5
