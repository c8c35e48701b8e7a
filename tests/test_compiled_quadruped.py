"""The compiled quadruped against values derived here without the model
compiler: the oracle steps the compiler's model dump, so a wrong mass,
inertia, mixed contact parameter or invweight in the compiler would reach
both sides of every parity test.  Each quantity is recomputed from the MJCF
text's numbers and the mechanics:

  * body masses and inertia tensors about the body COM: the uniform-density
    solids (box, capsule, sphere) integrated numerically over their volume,
    combined with the parallel-axis theorem;
  * the 79 candidate pairs' mixed contact parameters: MuJoCo's documented
    defaults (friction 1 / 0.005 / 0.0001, solref 0.02 1, solimp 0.9 0.95
    0.001 0.5 2), every geom sharing them, so the mixture is the default;
  * position actuators: gain kp, bias (0, -kp, -kv), control range = joint
    range;
  * meaninertia = trace(M) / nv, dof_invweight0 = diag(M^-1) (averaged over
    the translational / rotational dofs of the free joint) and
    body_invweight0 = mean diagonal of J M^-1 J' (translation, rotation; J
    at the body COM), with M, cdof and the COMs taken from the FP64
    oracle's own kinematics and CRBA at qpos0 (oracle/o_dyn.c), not from
    the compiler's;
  * each pair's invweights = the sum of its two bodies' body_invweight0.
"""
import ctypes as C

import numpy as np
import pytest

import mjb200
import oracle

L, R_CAP, R_FOOT = 0.213, 0.02, 0.022


def capsule_inertia(mass, r, half, n=200001):
    """Solid capsule along z centred at 0 (cylinder half-length `half`,
    radius r): (I_perp, I_axial) about its centre, by integrating thin disks
    over z (Simpson's rule)."""
    z = np.linspace(-(half + r), half + r, n)
    a2 = np.where(np.abs(z) <= half, r * r, np.maximum(r * r - (np.abs(z) - half) ** 2, 0.0))
    dz = z[1] - z[0]
    w = np.ones(n)
    w[1:-1:2], w[2:-1:2] = 4, 2
    w *= dz / 3
    area = np.pi * a2
    vol = np.sum(w * area)
    rho = mass / vol
    i_ax = rho * np.sum(w * area * a2 / 2)
    i_perp = rho * np.sum(w * area * (a2 / 4 + z * z))
    return i_perp, i_ax


def box_inertia(mass, a, b, c):
    return np.diag([mass / 3 * (b * b + c * c), mass / 3 * (a * a + c * c), mass / 3 * (a * a + b * b)])


def body_tensor(d, b):
    """Inertia tensor about the COM in the body frame from the dump's
    (body_iquat, body_inertia), and the COM body_ipos."""
    q = d["body_iquat"].reshape(-1, 4)[b]
    w, x, y, z = q / np.linalg.norm(q)
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    return R @ np.diag(d["body_inertia"].reshape(-1, 3)[b]) @ R.T, d["body_ipos"].reshape(-1, 3)[b]


@pytest.fixture(scope="module")
def dump(quad_model):
    return quad_model.dump()


def test_masses_and_inertias_from_the_solids(dump):
    d = dump
    names = ["world", "trunk"] + [f"{leg}_{part}" for leg, _, _ in mjb200.models.QUAD_LEGS for part in ("hip", "thigh", "calf")]
    mass = d["body_mass"]
    i_perp, i_ax = capsule_inertia(0.7, R_CAP, L / 2)
    for b, nm in enumerate(names):
        if b == 0:
            continue
        I, com = body_tensor(d, b)
        if nm == "trunk":
            want_m, want_com, want_I = 6.0, np.zeros(3), box_inertia(6.0, 0.19, 0.05, 0.04)
        elif nm.endswith("hip"):
            want_m, want_com, want_I = 0.5, np.zeros(3), np.diag([3e-4] * 3)
        elif nm.endswith("thigh"):
            want_m, want_com, want_I = 0.7, np.array([0, 0, -L / 2]), np.diag([i_perp, i_perp, i_ax])
        else:
            # capsule (COM at -L/2) and the foot sphere (at -L), about their joint COM
            mc, ms = 0.7, 0.05
            zc = (mc * (-L / 2) + ms * (-L)) / (mc + ms)
            dc, ds = -L / 2 - zc, -L - zc
            isph = 0.4 * ms * R_FOOT ** 2
            want_m, want_com = mc + ms, np.array([0, 0, zc])
            want_I = np.diag([i_perp + mc * dc * dc + isph + ms * ds * ds, i_perp + mc * dc * dc + isph + ms * ds * ds, i_ax + isph])
        assert mass[b] == pytest.approx(want_m, rel=1e-9), nm
        np.testing.assert_allclose(com, want_com, atol=1e-9, err_msg=nm)
        np.testing.assert_allclose(I, want_I, rtol=1e-6, atol=1e-12, err_msg=nm)


def test_mixed_contact_parameters_are_the_defaults(dump):
    d = dump
    pr = d["pair_real"].reshape(-1, 16)
    pi = d["pair_int"].reshape(-1, 6)
    assert len(pr) == 79
    np.testing.assert_allclose(pr[:, 0:2], 0.0)                                   # margin, gap
    np.testing.assert_allclose(pr[:, 2:7], np.tile([1.0, 1.0, 0.005, 0.0001, 0.0001], (79, 1)))   # friction per direction
    np.testing.assert_allclose(pr[:, 7:9], np.tile([0.02, 1.0], (79, 1)))          # solref
    np.testing.assert_allclose(pr[:, 9:14], np.tile([0.9, 0.95, 0.001, 0.5, 2.0], (79, 1)))      # solimp
    assert np.all(pi[:, 4] == 3)                                                   # condim


def test_position_actuators(dump):
    d = dump
    gain = d["actuator_gainprm"].reshape(-1, 3)
    bias = d["actuator_biasprm"].reshape(-1, 3)
    crange = d["actuator_ctrlrange"].reshape(-1, 2)
    rng = d["jnt_range"].reshape(-1, 2)
    trn = d["actuator_trnid"]
    assert len(gain) == 12
    np.testing.assert_allclose(gain[:, 0], 20.0)
    np.testing.assert_allclose(bias, np.tile([0.0, -20.0, -0.5], (12, 1)))
    np.testing.assert_allclose(crange, rng[trn])
    np.testing.assert_allclose(d["dof_armature"], [0.0] * 6 + [0.01] * 12)


def _oracle_qpos0(dump):
    om = oracle.OracleModel(dump)
    env = oracle.OracleEnv(om)
    env.a["qpos"][:] = dump["qpos0"]
    env.a["qvel"][:] = 0
    oracle.lib.oracle_kinematics(C.byref(om.c), C.byref(env.d))
    oracle.lib.oracle_com(C.byref(om.c), C.byref(env.d), None)
    oracle.lib.oracle_crb(C.byref(om.c), C.byref(env.d), None)
    return om, env


def test_meaninertia_and_invweights_from_the_oracle(dump):
    d = dump
    om, env = _oracle_qpos0(d)
    nv, nb = om.nv, om.nbody
    M = env.a["M"].reshape(nv, nv)
    Minv = np.linalg.inv(M)
    assert d["opt_real"][7] == pytest.approx(np.trace(M) / nv, rel=1e-9)           # meaninertia
    dv = np.diag(Minv).copy()
    want = np.concatenate([[dv[:3].mean()] * 3, [dv[3:6].mean()] * 3, dv[6:]])
    np.testing.assert_allclose(d["dof_invweight0"], want, rtol=1e-9)
    cdof = env.a["cdof"].reshape(nv, 6)
    scom = env.a["subtree_com"].reshape(nb, 3)
    xipos = env.a["xipos"].reshape(nb, 3)
    root = d["body_rootid"]
    dofb = d["dof_bodyid"]
    sub = d["body_subtreesize"]
    biw = d["body_invweight0"].reshape(nb, 2)
    for b in range(1, nb):
        off = xipos[b] - scom[root[b]]
        J = np.zeros((6, nv))
        for i in range(nv):
            if not (dofb[i] <= b < dofb[i] + sub[dofb[i]]):
                continue
            ang, lin = cdof[i, :3], cdof[i, 3:]
            J[:3, i] = lin + np.cross(ang, off)
            J[3:, i] = ang
        A = np.diag(J @ Minv @ J.T)
        assert biw[b, 0] == pytest.approx(A[:3].mean(), rel=1e-9), b
        assert biw[b, 1] == pytest.approx(A[3:].mean(), rel=1e-9), b
    pr = d["pair_real"].reshape(-1, 16)
    pi = d["pair_int"].reshape(-1, 6)
    np.testing.assert_allclose(pr[:, 14], biw[pi[:, 2], 0] + biw[pi[:, 3], 0], rtol=1e-12)
    np.testing.assert_allclose(pr[:, 15], biw[pi[:, 2], 1] + biw[pi[:, 3], 1], rtol=1e-12)
