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
    Christoffel term  dM/dt v - 1/2 d(v' M v)/dq,  from differences of M.

These do not involve the kernels, the compiler's inertia formulas (the
body inertias are read from the same dump the oracle uses) or any MuJoCo
code: they check the recursions (forward.hpp:143-397 of the reference) by
an independent route.
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
