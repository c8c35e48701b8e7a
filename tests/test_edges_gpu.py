"""Edge cases of the batched step against the FP64 oracle or against exact
expectations: contact / row overflow with tiny capacities (the same contacts
kept and the same status bits), bad-state reset, masked reset, actuator-gain
randomisation and the implicitfast integrator.

Tolerances as in the quadruped parity test (qacc relative error <= 2e-3 per
env, <= 1e-4 median; qpos / qvel after one step within 1e-5 / 1e-4)."""
import ctypes as C

import numpy as np
import pytest

import mjb200
import oracle
from parity import contact_sets_match, gpu_step_from, oracle_step_from, rel_err
from test_parity_gpu import visited_states

pytestmark = pytest.mark.gpu


def test_overflow_keeps_same_contacts_as_oracle(quad_model):
    """ncon_max 2 / nefc_max 10: contacts past the capacity and the first
    row group that does not fit are dropped with the same rule on both
    sides; status bits 4 (contacts) and 8 (rows) agree."""
    om = oracle.OracleModel(quad_model.dump())
    B = 32
    (qp, qv, ctrl), = visited_states(om, nsteps=(60,), B=B)
    sim = mjb200.BatchedSim(quad_model, B, ncon_max=2, nefc_max=10)
    g = gpu_step_from(sim, qp, qv, ctrl, 2, 10)
    o = oracle_step_from(om, qp.astype(np.float64), qv.astype(np.float64), ctrl.astype(np.float64), ncon_max=2, nefc_max=10)
    flagged = 0
    errs = []
    for e in range(B):
        st = g["stats"]
        assert st["status"][e] == o[e]["status"], (e, st["status"][e], o[e]["status"])
        flagged += st["status"][e] != 0
        ok, nb = contact_sets_match(g["con"][e], o[e]["contacts"], st["ncon"][e])
        assert ok
        if nb == 0:
            assert st["ncon"][e] == o[e]["ncon"] and st["nefc"][e] == o[e]["nefc"]
            errs.append(rel_err(g["vec"][e, 2, : om.nv], o[e]["qacc"]))
    assert flagged > 0
    assert np.median(errs) <= 1e-4 and max(errs) <= 2e-3


def test_bad_state_resets_only_that_env(quad_model):
    B = 16
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=33)
    q = q.astype(np.float32)
    v = v.astype(np.float32)
    ctrl = mjb200.models.quadruped_controls_fast(B, 0, seed=34).astype(np.float32)
    bad = q.copy()
    bad[3, 9] = np.nan
    bad[11, 2] = np.inf
    a = mjb200.BatchedSim(quad_model, B)
    a.set_state(bad, v)
    a.step(ctrl, 1)
    st = a.stats()
    assert st["status"][3] & 1 and st["status"][11] & 1
    assert np.all(np.delete(st["status"], [3, 11]) == 0)
    qa, va = a.state()
    # the reset envs stepped from qpos0 with zero velocity (and zero warm start)
    q0 = quad_model.dump()["qpos0"].astype(np.float32)
    ref_q = q.copy()
    ref_v = v.copy()
    ref_q[[3, 11]] = q0
    ref_v[[3, 11]] = 0
    b = mjb200.BatchedSim(quad_model, B)
    b.set_state(ref_q, ref_v)
    b.step(ctrl, 1)
    qb, vb = b.state()
    assert np.array_equal(qa, qb) and np.array_equal(va, vb)


def test_masked_reset(quad_model):
    B = 24
    sim = mjb200.BatchedSim(quad_model, B)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=35)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    for c in range(4):
        sim.step(mjb200.models.quadruped_controls_fast(B, c, seed=36).astype(np.float32), 4)
    before_q, before_v = sim.state()
    mask = np.zeros(B, np.int32)
    mask[[0, 5, 23]] = 1
    sim.reset(mask)
    qp, qv = sim.state()
    q0 = quad_model.dump()["qpos0"].astype(np.float32)
    assert np.array_equal(qp[mask == 1], np.tile(q0, (3, 1))) and not qv[mask == 1].any()
    assert np.array_equal(qp[mask == 0], before_q[mask == 0]) and np.array_equal(qv[mask == 0], before_v[mask == 0])


def test_gain_randomisation_parity(quad_model):
    om = oracle.OracleModel(quad_model.dump())
    B = 24
    (qp, qv, ctrl), = visited_states(om, nsteps=(40,), B=B)
    sim = mjb200.BatchedSim(quad_model, B, domain_rand=1)
    rng = np.random.default_rng(4)
    gain = rng.uniform(0.7, 1.3, size=(B, quad_model.nu)).astype(np.float32)
    assert sim.set_env_params(gain_scale=gain) == 0
    g = gpu_step_from(sim, qp, qv, ctrl, 64, 256)
    errs = []
    for e in range(B):
        env = oracle.OracleEnv(om)
        env.a["qpos"][:] = qp[e]
        env.a["qvel"][:] = qv[e]
        env.a["ctrl"][: om.nu] = ctrl[e]
        gs = np.ascontiguousarray(gain[e], np.float64)
        env.step(0, oracle.ORand(None, 1.0, gs.ctypes.data_as(C.POINTER(C.c_double))))
        errs.append(rel_err(g["vec"][e, 2, : om.nv], env.a["qacc"]))
        assert np.abs(g["qpos"][e] - env.a["qpos"]).max() < 1e-5
    assert np.median(errs) <= 1e-4 and max(errs) <= 2e-3


def test_implicitfast_integrator_parity():
    xml = mjb200.models.quadruped_xml().replace('integrator="Euler"', 'integrator="implicitfast"')
    model = mjb200.load_model_from_string(xml)
    om = oracle.OracleModel(model.dump())
    B = 24
    states = visited_states(om, nsteps=(30,), B=B)
    sim = mjb200.BatchedSim(model, B, integrator=3)
    for qp, qv, ctrl in states:
        g = gpu_step_from(sim, qp, qv, ctrl, 64, 256)
        o = oracle_step_from(om, qp.astype(np.float64), qv.astype(np.float64), ctrl.astype(np.float64))
        for e in range(B):
            assert np.abs(g["qpos"][e] - o[e]["qpos"]).max() < 1e-5
            assert np.abs(g["qvel"][e] - o[e]["qvel"]).max() < 1e-4 * max(1.0, np.abs(o[e]["qvel"]).max())


def test_gravcomp_com_offset_drag_parity():
    """Gravity compensation on the thighs (gravcomp 0.6), per-env COM offsets
    (U[-1, 1] cm per body, body frame) and per-env quadratic drag on the
    trunk's free joint (k U[0, 3]) against the oracle at visited states."""
    xml = mjb200.models.quadruped_xml().replace('_thigh" pos=', '_thigh" gravcomp="0.6" pos=')
    assert xml.count('gravcomp="0.6"') == 4
    model = mjb200.load_model_from_string(xml)
    om = oracle.OracleModel(model.dump())
    B = 24
    (qp, qv, ctrl), = visited_states(om, nsteps=(40,), B=B)
    sim = mjb200.BatchedSim(model, B, domain_rand=1)
    nb = int(model.dump()["sizes"][3])
    rng = np.random.default_rng(21)
    cd = rng.uniform(-0.01, 0.01, size=(B, nb, 3)).astype(np.float32)
    cd[:, 0] = 0
    drag = rng.uniform(0, 3, size=(B, 1)).astype(np.float32)
    assert sim.set_env_params(com_delta=cd) == 0
    assert sim.set_free_drag(drag) == 0
    qv = qv.copy()
    qv[:, :3] += rng.normal(0, 1.0, size=(B, 3)).astype(np.float32)   # drag needs a moving trunk
    g = gpu_step_from(sim, qp, qv, ctrl, 64, 256)
    errs = []
    for e in range(B):
        env = oracle.OracleEnv(om)
        env.a["qpos"][:] = qp[e]
        env.a["qvel"][:] = qv[e]
        env.a["ctrl"][: om.nu] = ctrl[e]
        c64 = np.ascontiguousarray(cd[e].astype(np.float64).reshape(-1))
        k64 = np.ascontiguousarray(drag[e].astype(np.float64))
        rand = oracle.ORand(None, 1.0, None, c64.ctypes.data_as(C.POINTER(C.c_double)), k64.ctypes.data_as(C.POINTER(C.c_double)))
        env.step(0, rand)
        assert g["stats"]["status"][e] == 0 and env.d.status == 0
        errs.append(rel_err(g["vec"][e, 2, : om.nv], env.a["qacc"]))
        assert np.abs(g["qpos"][e] - env.a["qpos"]).max() < 1e-5
    assert np.median(errs) <= 1e-4 and max(errs) <= 2e-3, (np.median(errs), max(errs))
    # the three terms change the step: without them the accelerations differ
    plain = mjb200.BatchedSim(mjb200.load_model_from_string(mjb200.models.quadruped_xml()), B)
    gp = gpu_step_from(plain, qp, qv, ctrl, 64, 256)
    assert np.abs(gp["vec"][:, 2] - g["vec"][:, 2]).max() > 1e-2


def test_batched_grad_step_matches_oracle_differences(quad_model):
    """mjmlx_batched_grad_step: d(qvel after one step)/d(ctrl) by central
    differences on the GPU against the same differences of the FP64 oracle
    (FP32 steps resolve the 1e-3 control perturbation to about 1e-3 of the
    Jacobian's scale); the state and controls are restored."""
    om = oracle.OracleModel(quad_model.dump())
    B = 8
    (qp, qv, ctrl), = visited_states(om, nsteps=(40,), B=B)
    sim = mjb200.BatchedSim(quad_model, B)
    sim.set_state(qp, qv)
    sim.step(ctrl, 1)
    q1, v1 = sim.state()
    G = sim.grad_step()
    q2, v2 = sim.state()
    assert np.array_equal(q1, q2) and np.array_equal(v1, v2)
    nv, nu = om.nv, om.nu
    for e in range(B):
        ref = np.zeros((nv, nu))
        for j in range(nu):
            h = 1e-3 * max(1.0, abs(float(ctrl[e, j])))
            vs = []
            for sg in (1, -1):
                env = oracle.OracleEnv(om)
                env.a["qpos"][:] = q1[e]
                env.a["qvel"][:] = v1[e]
                c = ctrl[e].astype(np.float64).copy()
                c[j] += sg * np.float32(h)
                env.a["ctrl"][:nu] = c.astype(np.float32)
                env.step()
                vs.append(env.a["qvel"].copy())
            ref[:, j] = (vs[0] - vs[1]) / (2 * h)
        assert np.abs(G[e] - ref).max() <= 2e-2 * np.abs(ref).max(), (e, np.abs(G[e] - ref).max(), np.abs(ref).max())
