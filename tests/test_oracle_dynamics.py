"""The oracle's CRBA mass matrix and RNE bias force against the Lagrangian
mechanics of its own forward kinematics (CPU only).

Every body's COM velocity and angular velocity Jacobian is taken by central
differences of the oracle's forward kinematics (xipos, ximat) along each
dof, the configuration moved by the joints' own integration map (free and
ball joints: the quaternion times the exponential of a body-frame rotation).
From those Jacobians alone:

  * M = sum over bodies of m Jv' Jv + Jw' I_world Jw, plus the armature on
    the diagonal, must equal the composite-rigid-body M;
  * at zero velocity the bias force is the gradient of the potential
    energy, sum over bodies of m g Jv_z;
  * for a fixed-base chain (hinges and slides only, where the coordinates
    are ordinary ones) the velocity part of the bias force is the
    Christoffel term  dM/dt v - 1/2 d(v' M v)/dq,  from differences of M;
  * each contact's pyramid rows are the normal and tangential components
    of the relative velocity of the contact point on the two bodies, and
    the normal row is the gradient of the contact distance.

These do not involve the kernels, the compiler's inertia formulas (the
body inertias are read from the same dump the oracle uses) or any MuJoCo
code: they check the recursions (forward.hpp:143-397 of the reference)
and the contact Jacobians (solver.hpp:474-571) by an independent route.
"""
import ctypes as C

import numpy as np
import pytest

import mjb200
import oracle

G = 9.81
EPS = 1e-6


def quat_mul(a, b):
    w1, x1, y1, z1 = a
    w2, x2, y2, z2 = b
    return np.array([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2])


def quat_exp(w):
    a = np.linalg.norm(w)
    if a < 1e-300:
        return np.array([1.0, 0, 0, 0])
    return np.concatenate([[np.cos(a / 2)], np.sin(a / 2) * w / a])


def integrate(d, q, v):
    """q moved by the velocity-space step v (one unit of time)."""
    q = q.copy()
    for j, t in enumerate(d["jnt_type"]):
        qa, va = d["jnt_qposadr"][j], d["jnt_dofadr"][j]
        if t == 0:
            q[qa:qa + 3] += v[va:va + 3]
            q[qa + 3:qa + 7] = quat_mul(q[qa + 3:qa + 7], quat_exp(v[va + 3:va + 6]))
        elif t == 1:
            q[qa:qa + 4] = quat_mul(q[qa:qa + 4], quat_exp(v[va:va + 3]))
        else:
            q[qa] += v[va]
    return q


class Probe:
    def __init__(self, xml):
        self.d = mjb200.load_model_from_string(xml).dump()
        self.om = oracle.OracleModel(self.d)
        self.env = oracle.OracleEnv(self.om, 64, 256)
        self.nv, self.nb = self.om.nv, self.om.nbody

    def fk(self, q):
        self.env.a["qpos"][:] = q
        oracle.lib.oracle_kinematics(C.byref(self.om.c), C.byref(self.env.d))
        return self.env.a["xipos"].reshape(self.nb, 3).copy(), self.env.a["ximat"].reshape(self.nb, 3, 3).copy()

    def dynamics(self, q, v):
        """(M, qfrc_bias) of the oracle's CRBA / RNE at (q, v)."""
        e = self.env
        e.a["qpos"][:] = q
        e.a["qvel"][:] = v
        for fn in ("oracle_kinematics",):
            getattr(oracle.lib, fn)(C.byref(self.om.c), C.byref(e.d))
        for fn in ("oracle_com", "oracle_crb", "oracle_rne"):
            getattr(oracle.lib, fn)(C.byref(self.om.c), C.byref(e.d), None)
        return e.a["M"].reshape(self.nv, self.nv).copy(), e.a["qfrc_bias"].copy()

    def jacobians(self, q):
        """Jv[b] (3 x nv) and Jw[b] (3 x nv, world frame) by central
        differences of the forward kinematics."""
        nv, nb = self.nv, self.nb
        Jv = np.zeros((nb, 3, nv))
        Jw = np.zeros((nb, 3, nv))
        for i in range(nv):
            e = np.zeros(nv)
            e[i] = EPS
            p1, R1 = self.fk(integrate(self.d, q, e))
            p0, R0 = self.fk(integrate(self.d, q, -e))
            Jv[:, :, i] = (p1 - p0) / (2 * EPS)
            for b in range(nb):
                W = (R1[b] @ R0[b].T - R0[b] @ R1[b].T) / (4 * EPS)     # skew part of dR R'
                Jw[b, :, i] = [W[2, 1], W[0, 2], W[1, 0]]
        return Jv, Jw

    def lagrange_mass(self, q):
        Jv, Jw = self.jacobians(q)
        _, R = self.fk(q)
        inert = self.d["body_inertia"].reshape(-1, 3)
        mass = self.d["body_mass"]
        M = np.diag(self.d["dof_armature"]).astype(float)
        for b in range(1, self.nb):
            Iw = R[b] @ np.diag(inert[b]) @ R[b].T
            M += mass[b] * Jv[b].T @ Jv[b] + Jw[b].T @ Iw @ Jw[b]
        return M, Jv

    def gravity_force(self, Jv):
        mass = self.d["body_mass"]
        return sum(mass[b] * G * Jv[b][2] for b in range(1, self.nb))


def random_pose(d, rng, scale=0.5):
    q = d["qpos0"].astype(float).copy()
    return integrate(d, q, rng.uniform(-scale, scale, size=len(d["dof_armature"])))


@pytest.mark.parametrize("name", ["quadruped", "humanoid", "arm"])
def test_crba_mass_matrix_and_gravity_from_the_lagrangian(name):
    xml = {"quadruped": mjb200.models.quadruped_xml, "humanoid": mjb200.models.humanoid_xml, "arm": mjb200.models.arm_xml}[name]()
    p = Probe(xml)
    rng = np.random.default_rng(11)
    for _ in range(3):
        q = random_pose(p.d, rng)
        M_lag, Jv = p.lagrange_mass(q)
        M, bias0 = p.dynamics(q, np.zeros(p.nv))
        scale = np.abs(M).max()
        np.testing.assert_allclose(M, M_lag, atol=1e-7 * scale, err_msg=name)
        np.testing.assert_allclose(bias0, p.gravity_force(Jv), atol=1e-7 * max(1.0, np.abs(bias0).max()), err_msg=name)


def test_rne_velocity_terms_from_the_christoffel_symbols():
    """The arm with its free object at rest: hinges and slides only move,
    so d/dt (dL/dv) - dL/dq in ordinary coordinates gives the bias force
    C(q, v) v = dM/dt v - 1/2 grad_q (v' M v) + gravity."""
    p = Probe(mjb200.models.arm_xml())
    d = p.d
    rng = np.random.default_rng(5)
    arm = np.array([d["jnt_type"][d["dof_jntid"][i]] in (2, 3) for i in range(p.nv)])
    h = 1e-5
    for _ in range(3):
        q = random_pose(d, rng, 0.4)
        v = np.where(arm, rng.uniform(-2.0, 2.0, size=p.nv), 0.0)
        Mp, _ = p.dynamics(integrate(d, q, h * v), np.zeros(p.nv))
        Mm, _ = p.dynamics(integrate(d, q, -h * v), np.zeros(p.nv))
        Mdot_v = (Mp - Mm) @ v / (2 * h)
        grad = np.zeros(p.nv)
        for i in np.flatnonzero(arm):
            e = np.zeros(p.nv)
            e[i] = h
            Ap, _ = p.dynamics(integrate(d, q, e), np.zeros(p.nv))
            Am, _ = p.dynamics(integrate(d, q, -e), np.zeros(p.nv))
            grad[i] = v @ (Ap - Am) @ v / (2 * h)
        _, bias0 = p.dynamics(q, np.zeros(p.nv))
        _, bias = p.dynamics(q, v)
        want = Mdot_v - 0.5 * grad
        np.testing.assert_allclose((bias - bias0)[arm], want[arm], atol=1e-6 * max(1.0, np.abs(want).max()))
        assert np.abs(want[arm]).max() > 0.1          # the velocity terms are not negligible here


def skew(r):
    return np.array([[0, -r[2], r[1]], [r[2], 0, -r[0]], [-r[1], r[0], 0]])


def test_contact_rows_from_the_motion_of_the_contact_point():
    """The pyramid rows of every contact (reference solver.hpp:474-571)
    against the material velocity of the contact point on each body, from
    the finite-difference Jacobians: with Jrel = J_point(body2) -
    J_point(body1), J_point = Jv - [p - xipos]x Jw, the rows' mean is
    n' Jrel and their half-difference over mu is t' Jrel; the normal row is
    also the gradient of the contact distance (same contacts, moved
    configuration)."""
    xml = ('<mujoco><option timestep="0.002"/><worldbody><geom type="plane" size="5 5 0.1"/>'
           '<body pos="0 0 0.098"><freejoint/><geom type="sphere" size="0.1" mass="1"/></body>'
           '<body pos="0.5 0 0.045" euler="0.3 0.2 0"><freejoint/><geom type="capsule" size="0.05 0.2" euler="0 1.5 0" mass="1"/></body>'
           '<body pos="-0.5 0 0.097" euler="0.02 -0.03 0.4"><freejoint/><geom type="box" size="0.1 0.15 0.1" mass="2"/></body>'
           '<body pos="0 0.6 0.3"><freejoint/><geom type="sphere" size="0.1" mass="1"/></body>'
           '<body pos="0.05 0.62 0.49"><freejoint/><geom type="sphere" size="0.1" mass="0.5"/></body>'
           '</worldbody></mujoco>')
    p = Probe(xml)
    d, om, env = p.d, p.om, p.env
    rng = np.random.default_rng(3)
    q = d["qpos0"].astype(float).copy()

    def contacts_at(qq):
        env.a["qpos"][:] = qq
        env.a["qvel"][:] = 0
        oracle.lib.oracle_kinematics(C.byref(om.c), C.byref(env.d))
        for fn in ("oracle_com", "oracle_crb", "oracle_rne"):
            getattr(oracle.lib, fn)(C.byref(om.c), C.byref(env.d), None)
        oracle.lib.oracle_collide(C.byref(om.c), C.byref(env.d))
        oracle.lib.oracle_make_constraints(C.byref(om.c), C.byref(env.d), None)
        return env.contacts(), env.efc()

    con, efc = contacts_at(q)
    gtype = d["geom_type"]
    kinds = {(int(gtype[int(c[14])]), int(gtype[int(c[15])])) for c in con}
    assert kinds == {(0, 2), (0, 3), (0, 6), (2, 2)} and len(con) >= 6
    _, R = p.fk(q)
    xipos, _ = p.fk(q)
    Jv, Jw = p.jacobians(q)
    gbody = d["geom_bodyid"]
    pr = d["pair_real"].reshape(-1, 16)
    for c in con:
        pos, n, t1, t2 = c[0:3], c[3:6], c[6:9], c[9:12]
        b1, b2 = gbody[int(c[14])], gbody[int(c[15])]

        def jpoint(b):
            if b == 0:
                return np.zeros((3, p.nv))
            return Jv[b] - skew(pos - xipos[b]) @ Jw[b]

        Jrel = jpoint(b2) - jpoint(b1)
        r = int(c[19])
        J = efc["J"][r:r + 4]
        mu = pr[int(c[13]), 2:4]
        scale = max(1.0, np.abs(J).max())
        np.testing.assert_allclose((J[0] + J[1]) / 2, n @ Jrel, atol=1e-7 * scale)
        np.testing.assert_allclose((J[0] - J[1]) / (2 * mu[0]), t1 @ Jrel, atol=1e-7 * scale / mu[0])
        np.testing.assert_allclose((J[2] - J[3]) / (2 * mu[1]), t2 @ Jrel, atol=1e-7 * scale / mu[1])
    # distance gradient of the contacts whose point is unique (sphere-plane,
    # sphere-sphere): along a random velocity direction
    v = rng.normal(size=p.nv)
    h = 1e-6
    cp, _ = contacts_at(integrate(d, q, h * v))
    cm, _ = contacts_at(integrate(d, q, -h * v))
    con, efc = contacts_at(q)
    checked = 0
    for k, c in enumerate(con):
        t = (gtype[int(c[14])], gtype[int(c[15])])
        if t not in ((0, 2), (2, 2)):
            continue
        same = [i for i in range(len(cp)) if int(cp[i, 13]) == int(c[13])], [i for i in range(len(cm)) if int(cm[i, 13]) == int(c[13])]
        ddist = (cp[same[0][0], 12] - cm[same[1][0], 12]) / (2 * h)
        r = int(c[19])
        Jn = (efc["J"][r] + efc["J"][r + 1]) / 2
        assert Jn @ v == pytest.approx(ddist, rel=1e-6, abs=1e-8)
        checked += 1
    assert checked == 2                        # the floor sphere and the sphere pair


def mujoco_impedance(solref, solimp, pos, h, refsafe=True):
    """MuJoCo's documented soft-constraint parameters, written from its
    documentation: (k, b, imp) for signed distance pos."""
    tc, dr = solref
    dmin, dmax, width, mid, power = solimp
    dmin, dmax = np.clip([dmin, dmax], 1e-4, 0.9999)
    mid = np.clip(mid, 1e-4, 0.9999)
    power = max(power, 1.0)
    width = max(width, 1e-12)
    if tc > 0:
        if refsafe:
            tc = max(tc, 2 * h)
        k = 1 / (dmax * dmax * tc * tc * dr * dr)
        b = 2 / (dmax * tc)
    else:
        k, b = -tc / (dmax * dmax), -dr / dmax
    x = abs(pos) / width
    if x >= 1:
        imp = dmax
    else:
        y = x ** power / mid ** (power - 1) if x < mid else 1 - (1 - x) ** power / (1 - mid) ** (power - 1)
        imp = dmin + y * (dmax - dmin)
    return k, b, imp


@pytest.mark.parametrize("solref,solimp,q,v", [
    ((0.02, 1.0), (0.9, 0.95, 0.001, 0.5, 2), 0.7, 0.3),      # defaults, deep
    ((0.02, 1.0), (0.9, 0.95, 0.1, 0.5, 2), 0.52, -0.4),      # inside the width, below mid
    ((0.02, 1.0), (0.5, 0.99, 0.1, 0.3, 3), 0.58, 0.1),       # inside the width, above mid, power 3
    ((0.001, 0.5), (0.9, 0.95, 0.001, 0.5, 2), 0.6, 0.0),     # time constant below 2 h: clamped
    ((-2000.0, -30.0), (0.9, 0.95, 0.001, 0.5, 2), 0.6, 0.2),  # direct stiffness and damping
])
def test_limit_row_impedance_follows_the_documented_formulas(solref, solimp, q, v):
    """A hinge past its upper limit 0.5: the limit row's D = imp / ((1 - imp)
    invweight) and aref = -b J v - k imp pos with pos = 0.5 - q, against
    MuJoCo's documented solref / solimp semantics restated above
    (reference solver.hpp:122-138, 347-368)."""
    h = 0.002
    xml = (f'<mujoco><compiler angle="radian"/><option timestep="{h}"/><worldbody><body><joint type="hinge" axis="0 1 0" limited="true" range="-0.5 0.5" '
           f'solreflimit="{solref[0]} {solref[1]}" solimplimit="{" ".join(str(x) for x in solimp)}"/>'
           '<geom type="capsule" fromto="0 0 0 0.3 0 0" size="0.03" mass="1"/></body></worldbody></mujoco>')
    p = Probe(xml)
    env = p.env
    env.a["qpos"][0] = q
    env.a["qvel"][0] = v
    env.step()
    e = p.env.efc()
    assert list(e["type"]) == [1]
    pos = 0.5 - q
    k, b, imp = mujoco_impedance(solref, solimp, pos, h)
    invw = p.d["dof_invweight0"][0]
    assert e["J"][0, 0] == -1.0
    assert e["D"][0] == pytest.approx(imp / ((1 - imp) * invw), rel=1e-12)
    assert e["aref"][0] == pytest.approx(-b * (-v) - k * imp * pos, rel=1e-12)
