"""Elliptic friction cones on the GPU against the FP64 oracle (MuJoCo's cone
model: one normal row and condim - 1 friction rows per contact, Newton with
the cone's zone-dependent Hessian).

Checked per env at states visited by oracle or GPU rollouts: row types in
order (normal 4, friction 6), D and aref within 1e-4 relative (FP32
impedance), row forces within 2e-3 of the largest force, qacc relative
error <= 1e-4 median and <= 2e-3 per env (5e-3 for general convex pairs,
whose FP32 normals on nearly parallel curved contacts carry a few 1e-4);
rollouts stay finite without resets.  The bin case is the 2048-env bin
workload with condim 6: contact pair lists equal on 64 sampled envs and
the same qacc bounds."""
import numpy as np
import pytest

import mjb200
import oracle
from parity import contact_sets_match, gpu_step_from, oracle_step_from, rel_err
from test_parity_gpu import visited_states

pytestmark = pytest.mark.gpu


def _box_states(om, B, seed):
    """States of the pushed box visited by oracle rollouts with pushes
    U[0, 10] N held for 10-200 steps (sticking and sliding)."""
    g = np.random.default_rng(seed)
    q = np.zeros((B, om.nq))
    v = np.zeros((B, om.nv))
    ctrl = np.zeros((B, 1))
    for e in range(B):
        env = oracle.OracleEnv(om)
        env.a["qpos"][:] = 0
        env.a["qpos"][2] = -0.0005
        env.a["qpos"][3] = 1
        push = g.uniform(0, 10)
        for t in range(int(g.integers(10, 200))):
            env.a["ctrl"][0] = push
            env.a["qvel"][1] += g.normal(0, 0.01)
            env.step()
        q[e], v[e], ctrl[e] = env.a["qpos"], env.a["qvel"], push
    return q.astype(np.float32), v.astype(np.float32), ctrl.astype(np.float32)


def _compare(g, o, B, nv, qtol=2e-3, rows=True):
    errs, ncone = [], 0
    for e in range(B):
        st = g["stats"]
        assert st["status"][e] == 0 and o[e]["status"] == 0
        n = o[e]["nefc"]
        assert st["nefc"][e] == n, (e, st["nefc"][e], n)
        ot = o[e]["efc"]["type"]
        assert list(g["efc"][e, :n, 0].astype(int)) == list(ot), e
        ncone += int((ot == 4).sum())
        if rows and n:
            np.testing.assert_allclose(g["efc"][e, :n, 2], o[e]["efc"]["D"], rtol=1e-4)
            aref = o[e]["efc"]["aref"]
            np.testing.assert_allclose(g["efc"][e, :n, 3], aref, rtol=1e-4, atol=1e-4 * np.abs(aref).max())
            f = o[e]["efc"]["force"]
            assert np.abs(g["efc"][e, :n, 1] - f).max() <= 2e-3 * max(1.0, np.abs(f).max()), e
        errs.append(rel_err(g["vec"][e, 2, :nv], o[e]["qacc"]))
    errs = np.array(errs)
    assert np.median(errs) <= 1e-4 and errs.max() <= qtol, (np.median(errs), errs.max())
    return ncone


@pytest.mark.parametrize("condim", [3, 4, 6])
@pytest.mark.parametrize("impratio", [1.0, 4.0])
def test_pushed_box_elliptic_parity(condim, impratio):
    model = mjb200.load_model_from_string(mjb200.models.pushed_box_xml("elliptic", condim, 0.5, impratio))
    om = oracle.OracleModel(model.dump())
    B = 32
    q, v, ctrl = _box_states(om, B, 10 * condim + int(impratio))
    sim = mjb200.BatchedSim(model, B, ncon_max=8, nefc_max=64)
    g = gpu_step_from(sim, q, v, ctrl, 8, 64)
    o = oracle_step_from(om, q.astype(np.float64), v.astype(np.float64), ctrl.astype(np.float64), ncon_max=8, nefc_max=64)
    assert _compare(g, o, B, om.nv) >= B


def test_pushed_box_elliptic_stick_and_slide_rollout():
    """On the GPU alone: below mu m g the box sticks, above it slides with
    every contact's friction on the cone boundary (|f_t| = mu f_n)."""
    model = mjb200.load_model_from_string(mjb200.models.pushed_box_xml("elliptic", 3))
    B = 2
    q = np.zeros((B, model.nq), np.float32)
    q[:, 2] = -0.0005
    q[:, 3] = 1
    sim = mjb200.BatchedSim(model, B, ncon_max=8, nefc_max=64)
    sim.set_state(q, np.zeros((B, model.nv), np.float32))
    ctrl = np.array([[3.0], [9.0]], np.float32)
    sim.step(ctrl, 200)
    qp, qv = sim.state()
    assert abs(qv[0, 0]) < 2e-3 and qv[1, 0] > 0.5
    # the sliding box hovers on and off the floor (the soft elliptic model's
    # sliding lift): sample 30 steps for contacts that carry load
    nlive = 0
    for t in range(30):
        g = gpu_step_from(sim, qp, qv, ctrl, 8, 64)
        qp, qv = g["qpos"], g["qvel"]
        n = g["stats"]["nefc"][1]
        f = g["efc"][1, :n, 1].reshape(-1, 3)
        live = f[:, 0] > 1e-3
        nlive += int(live.sum())
        if live.any():
            np.testing.assert_allclose(np.linalg.norm(f[live, 1:], axis=1), 0.5 * f[live, 0], rtol=1e-3)
    assert nlive > 0


def test_quadruped_elliptic_parity_and_rollout():
    model = mjb200.load_model_from_string(mjb200.models.quadruped_xml(cone="elliptic"))
    om = oracle.OracleModel(model.dump())
    B = 32
    states = visited_states(om, nsteps=(20, 60, 120), B=B)
    sim = mjb200.BatchedSim(model, B, ncon_max=48, nefc_max=160)
    ncone = 0
    for qp, qv, ctrl in states:
        g = gpu_step_from(sim, qp, qv, ctrl, 48, 160)
        o = oracle_step_from(om, qp.astype(np.float64), qv.astype(np.float64), ctrl.astype(np.float64), ncon_max=48, nefc_max=160)
        for e in range(B):
            ok, nb = contact_sets_match(g["con"][e], o[e]["contacts"], g["stats"]["ncon"][e])
            assert ok and nb == 0, e
        ncone += _compare(g, o, B, om.nv)
        for e in range(B):
            assert np.abs(g["qpos"][e] - o[e]["qpos"]).max() < 1e-5
    assert ncone > B
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=71)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    for c in range(30):
        sim.step(mjb200.models.quadruped_controls_fast(B, c, seed=72).astype(np.float32), 4)
    qp, qv = sim.state()
    assert np.isfinite(qp).all() and np.isfinite(qv).all() and np.all(sim.stats()["status"] == 0)


def test_convex_pile_elliptic_condim6_parity():
    model = mjb200.load_model_from_string(mjb200.models.convex_pile_xml(6, seed=2, condim=6, cone="elliptic"))
    om = oracle.OracleModel(model.dump())
    B = 32
    q, v = mjb200.models.box_pile_state(model, B, seed=9)
    ob = oracle.OracleBatch(om, B, 40, 240)
    ob.set_state(q, v)
    states = []
    for s in range(121):
        if s in (40, 120):
            qp, qv = ob.state()
            states.append((qp.astype(np.float32), qv.astype(np.float32)))
        ob.step(1, nthread=8)
    sim = mjb200.BatchedSim(model, B, ncon_max=40, nefc_max=240)
    for qp, qv in states:
        g = gpu_step_from(sim, qp, qv, None, 40, 240)
        o = oracle_step_from(om, qp.astype(np.float64), qv.astype(np.float64), np.zeros((B, 1)), ncon_max=40, nefc_max=240)
        keep = []
        for e in range(B):
            ok, nb = contact_sets_match(g["con"][e], o[e]["contacts"], g["stats"]["ncon"][e])
            assert ok, e
            if nb == 0:
                keep.append(e)
        assert len(keep) >= B - 2
        sub = {k: (val[keep] if k != "stats" else {kk: vv[keep] for kk, vv in val.items()}) for k, val in g.items()}
        _compare(sub, [o[e] for e in keep], len(keep), om.nv, qtol=5e-3, rows=False)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    sim.step(None, 300)
    qp, qv = sim.state()
    assert np.isfinite(qp).all() and np.all(sim.stats()["status"] == 0)


def test_bin_workload_elliptic_condim6_2048_envs_sampled_parity():
    """The bin workload with its cone: 2048 envs of 64 free convex bodies,
    condim 6, elliptic; 80 substeps from seeded poses, then one step checked
    on every 32nd env against the oracle (contact pairs, row counts and
    types, qacc)."""
    model = mjb200.load_model_from_string(mjb200.models.bin_xml(64, 1.0, seed=1, condim=6, cone="elliptic"))
    om = oracle.OracleModel(model.dump())
    B, ncon, nefc = 2048, 400, 2400
    q, v = mjb200.models.box_pile_state(model, B, seed=7)
    sim = mjb200.BatchedSim(model, B, ncon_max=ncon, nefc_max=nefc)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    sim.step(None, 80)
    qp, qv = sim.state()
    assert np.all(sim.stats()["status"] == 0) and np.isfinite(qp).all()
    g = gpu_step_from(sim, qp, qv, None, ncon, nefc)
    idx = np.arange(0, B, 32)
    o = oracle_step_from(om, qp[idx].astype(np.float64), qv[idx].astype(np.float64), np.zeros((len(idx), 1)), ncon_max=ncon, nefc_max=nefc)
    errs, flips, ncone = [], 0, 0
    for k, e in enumerate(idx):
        assert g["stats"]["status"][e] == 0 and o[k]["status"] == 0
        ok, nb = contact_sets_match(g["con"][e], o[k]["contacts"], g["stats"]["ncon"][e])
        assert ok, e
        flips += nb
        if nb == 0:
            n = o[k]["nefc"]
            assert g["stats"]["nefc"][e] == n
            assert list(g["efc"][e, :n, 0].astype(int)) == list(o[k]["efc"]["type"])
            ncone += int((o[k]["efc"]["type"] == 4).sum())
            errs.append(rel_err(g["vec"][e, 2, : om.nv], o[k]["qacc"]))
    errs = np.array(errs)
    print("sampled", len(idx), "boundary flips", flips, "cones", ncone, "median %.2e max %.2e" % (np.median(errs), errs.max()))
    assert len(errs) >= 60 and ncone > 0
    assert np.median(errs) <= 1e-4 and errs.max() <= 5e-3, (np.median(errs), errs.max())


def test_elliptic_cfrc_ext_is_the_contact_force_sum():
    """cfrc_ext's force part on the sliding box equals the sum over contacts
    of f_n n + f_1 t1 + f_2 t2 with the oracle's row forces and frames at
    the same state."""
    model = mjb200.load_model_from_string(mjb200.models.pushed_box_xml("elliptic", 3))
    om = oracle.OracleModel(model.dump())
    B = 8
    q, v, ctrl = _box_states(om, B, 5)
    sim = mjb200.BatchedSim(model, B, ncon_max=8, nefc_max=64, record=1)
    sim.set_state(q, v)
    sim.step(ctrl, 1)
    cf = sim.get("cfrc_ext").reshape(B, -1, 6)
    o = oracle_step_from(om, q.astype(np.float64), v.astype(np.float64), ctrl.astype(np.float64), ncon_max=8, nefc_max=64)
    checked = 0
    for e in range(B):
        F = np.zeros(3)
        f = o[e]["efc"]["force"].reshape(-1, 3)
        for c, con in enumerate(o[e]["contacts"]):
            F += f[c, 0] * con[3:6] + f[c, 1] * con[6:9] + f[c, 2] * con[9:12]
        if np.abs(F).max() < 1e-3:
            continue
        checked += 1
        got = cf[e, 1, 3:]
        err = min(np.abs(got - F).max(), np.abs(got + F).max())
        assert err <= 2e-3 * np.abs(F).max(), (e, got, F)
    assert checked >= B // 2
