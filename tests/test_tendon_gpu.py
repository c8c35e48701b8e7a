"""Fixed tendons on the GPU against the FP64 oracle: the tendon chain (five
fixed tendons with limits, frictionloss, springs with a dead band, a damper,
a tendon equality, a motor and a position actuator on tendons).

Checked per env, on random states that put tendons past their limits: row
types in order (equality, tendon frictionloss, tendon limits), each row's D
and aref, qfrc_smooth (passive + actuator - bias) and qacc; then a rollout
that stays finite, unflagged and holds the limit and the equality.

Tolerances: qfrc_smooth relative error <= 1e-5; D and aref within 1e-4
relative (FP32 impedance); qacc relative error <= 2e-3 per env and <= 1e-4
median, as in the quadruped parity test."""
import numpy as np
import pytest

import mjb200
import oracle
from parity import gpu_step_from, oracle_step_from, rel_err

pytestmark = pytest.mark.gpu

T0 = np.array([1.0, 0.5, 0, 0, 0, 0, 0, 0])
T3 = np.array([0, 0, 0, 0, 0, 0, 1.0, 0.7])
T4 = np.array([0, 0, 0, 0, 1.0, -0.3, 0, 0])


def _inputs(B, seed):
    g = np.random.default_rng(seed)
    q = g.normal(0.0, 0.45, size=(B, 8)).astype(np.float32)
    v = g.normal(0.0, 0.5, size=(B, 8)).astype(np.float32)
    ctrl = np.stack([g.uniform(-1, 1, B), g.uniform(-0.4, 0.4, B)], axis=1).astype(np.float32)
    return q, v, ctrl


def test_tendon_chain_single_step_parity():
    model = mjb200.load_model_from_string(mjb200.models.tendon_chain_xml(8))
    om = oracle.OracleModel(model.dump())
    B = 64
    q, v, ctrl = _inputs(B, 11)
    sim = mjb200.BatchedSim(model, B, ncon_max=4, nefc_max=32)
    g = gpu_step_from(sim, q, v, ctrl, 4, 32)
    o = oracle_step_from(om, q.astype(np.float64), v.astype(np.float64), ctrl.astype(np.float64), ncon_max=4, nefc_max=32)
    errs, nlim = [], 0
    for e in range(B):
        st = g["stats"]
        assert st["status"][e] == 0 and o[e]["status"] == 0
        n = o[e]["nefc"]
        assert st["nefc"][e] == n, (e, st["nefc"][e], n)
        ot = o[e]["efc"]["type"]
        gt = g["efc"][e, :n, 0].astype(int)
        assert list(gt) == list(ot), (e, gt, ot)
        nlim += int((ot == 1).sum())
        np.testing.assert_allclose(g["efc"][e, :n, 2], o[e]["efc"]["D"], rtol=1e-4)
        np.testing.assert_allclose(g["efc"][e, :n, 3], o[e]["efc"]["aref"], rtol=1e-4, atol=1e-4 * np.abs(o[e]["efc"]["aref"]).max())
        assert rel_err(g["vec"][e, 1, :8], o[e]["qfrc_smooth"]) <= 1e-5
        errs.append(rel_err(g["vec"][e, 2, :8], o[e]["qacc"]))
    assert nlim >= B // 4          # the states exercise tendon limits
    errs = np.array(errs)
    assert np.median(errs) <= 1e-4 and errs.max() <= 2e-3, (np.median(errs), errs.max())


def test_tendon_chain_rollout_holds_constraints():
    model = mjb200.load_model_from_string(mjb200.models.tendon_chain_xml(8))
    B = 32
    g = np.random.default_rng(12)
    q = g.normal(0.0, 0.1, size=(B, 8)).astype(np.float32)
    sim = mjb200.BatchedSim(model, B)
    sim.set_state(q, np.zeros_like(q))
    worst_lim, worst_eq = 0.0, 0.0
    for c in range(40):
        ctrl = np.stack([g.uniform(-1, 1, B), g.uniform(-0.4, 0.4, B)], axis=1).astype(np.float32)
        sim.step(ctrl, 25)
        qp, qv = sim.state()
        assert np.isfinite(qp).all() and np.isfinite(qv).all()
        if c > 1:
            worst_lim = max(worst_lim, float((np.abs(qp @ T0) - 0.3).max()))
            worst_eq = max(worst_eq, float(np.abs(qp @ T3 - 0.8 * (qp @ T4)).max()))
    assert np.all(sim.stats()["status"] == 0)
    assert worst_lim < 0.05 and worst_eq < 0.05, (worst_lim, worst_eq)


def test_tendon_overflow_rule_matches_oracle():
    """nefc_max 2: the equality row and one tendon frictionloss row fit; the
    second frictionloss row does not, so it and every limit row are dropped
    on both sides with status bit 8."""
    model = mjb200.load_model_from_string(mjb200.models.tendon_chain_xml(8))
    om = oracle.OracleModel(model.dump())
    B = 16
    q, v, ctrl = _inputs(B, 13)
    sim = mjb200.BatchedSim(model, B, ncon_max=4, nefc_max=2)
    g = gpu_step_from(sim, q, v, ctrl, 4, 2)
    o = oracle_step_from(om, q.astype(np.float64), v.astype(np.float64), ctrl.astype(np.float64), ncon_max=4, nefc_max=2)
    errs = []
    for e in range(B):
        assert g["stats"]["status"][e] == o[e]["status"] == 8
        assert g["stats"]["nefc"][e] == o[e]["nefc"] == 2
        errs.append(rel_err(g["vec"][e, 2, :8], o[e]["qacc"]))
    assert np.median(errs) <= 1e-4 and max(errs) <= 2e-3


def test_spatial_tendon_parity_and_rollout():
    """Spatial tendons (sphere and cylinder wrapping with a side site, a
    pulley, straight site pieces) on the wrapped arm: per env the row types
    in order, D and aref, qfrc_smooth and qacc against the oracle (same
    bounds as above), then a rollout under random motor commands that stays
    finite and unflagged."""
    model = mjb200.load_model_from_string(mjb200.models.spatial_tendon_xml())
    om = oracle.OracleModel(model.dump())
    B = 48
    g = np.random.default_rng(17)
    q = np.stack([g.uniform(-0.9, 0.9, B), g.uniform(-1.6, 1.6, B), g.uniform(-0.15, 0.15, B)], axis=1).astype(np.float32)
    v = g.normal(0, 1.0, size=(B, 3)).astype(np.float32)
    ctrl = np.stack([g.uniform(-1, 1, B), g.uniform(-0.1, 0.1, B)], axis=1).astype(np.float32)
    sim = mjb200.BatchedSim(model, B, ncon_max=4, nefc_max=32)
    gs = gpu_step_from(sim, q, v, ctrl, 4, 32)
    o = oracle_step_from(om, q.astype(np.float64), v.astype(np.float64), ctrl.astype(np.float64), ncon_max=4, nefc_max=32)
    errs, nlim = [], 0
    for e in range(B):
        assert gs["stats"]["status"][e] == 0 and o[e]["status"] == 0
        n = o[e]["nefc"]
        assert gs["stats"]["nefc"][e] == n
        ot = o[e]["efc"]["type"]
        assert list(gs["efc"][e, :n, 0].astype(int)) == list(ot)
        nlim += int((ot == 1).sum())
        np.testing.assert_allclose(gs["efc"][e, :n, 2], o[e]["efc"]["D"], rtol=1e-4)
        np.testing.assert_allclose(gs["efc"][e, :n, 3], o[e]["efc"]["aref"], rtol=1e-4, atol=1e-4 * np.abs(o[e]["efc"]["aref"]).max())
        assert rel_err(gs["vec"][e, 1, :3], o[e]["qfrc_smooth"]) <= 1e-5
        errs.append(rel_err(gs["vec"][e, 2, :3], o[e]["qacc"]))
    assert nlim > 0
    errs = np.array(errs)
    assert np.median(errs) <= 1e-4 and errs.max() <= 2e-3, (np.median(errs), errs.max())
    sim.set_state(q, v)
    for c in range(20):
        sim.step(np.stack([g.uniform(-1, 1, B), g.uniform(-0.1, 0.1, B)], axis=1).astype(np.float32), 25)
    qp, qv = sim.state()
    assert np.isfinite(qp).all() and np.isfinite(qv).all()
    assert np.all(sim.stats()["status"] == 0)
