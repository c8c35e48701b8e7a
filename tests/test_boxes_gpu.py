"""Box-box contacts (separating axes, clipped face contacts, edge-edge
contacts) on the GPU against the FP64 oracle: a pile of 4 free boxes of
seeded sizes dropped on a plane, single-step parity at states visited by an
oracle rollout (contact sets equal up to activation-boundary flips, row
counts equal, qacc relative error <= 2e-3 per env and <= 1e-4 median), and a
2 s rollout that stays finite without resets."""
import numpy as np
import pytest

import mjb200
import oracle
from parity import contact_sets_match, gpu_step_from, oracle_step_from, rel_err

pytestmark = pytest.mark.gpu


def test_box_pile_parity_and_rollout():
    model = mjb200.load_model_from_string(mjb200.models.box_pile_xml(4, seed=1))
    om = oracle.OracleModel(model.dump())
    B = 32
    q, v = mjb200.models.box_pile_state(model, B, seed=3)
    ob = oracle.OracleBatch(om, B, 64, 256)
    ob.set_state(q, v)
    states = []
    for s in range(121):
        if s in (20, 60, 120):
            qp, qv = ob.state()
            states.append((qp.astype(np.float32), qv.astype(np.float32)))
        ob.step(1, nthread=8)
    sim = mjb200.BatchedSim(model, B, ncon_max=32, nefc_max=160)
    nbb = 0
    for qp, qv in states:
        g = gpu_step_from(sim, qp, qv, None, 32, 160)
        o = oracle_step_from(om, qp.astype(np.float64), qv.astype(np.float64), np.zeros((B, 1)), ncon_max=32, nefc_max=160)
        errs = []
        for e in range(B):
            st = g["stats"]
            assert st["status"][e] == 0 and o[e]["status"] == 0
            ok, nb = contact_sets_match(g["con"][e], o[e]["contacts"], st["ncon"][e])
            assert ok, e
            nbb += int(sum(1 for c in o[e]["contacts"] if int(c[14]) > 0 and int(c[15]) > 0))
            if nb == 0:
                assert st["nefc"][e] == o[e]["nefc"]
                errs.append(rel_err(g["vec"][e, 2, : om.nv], o[e]["qacc"]))
        errs = np.array(errs)
        assert np.median(errs) <= 1e-4 and errs.max() <= 2e-3, (np.median(errs), errs.max())
    assert nbb > 0  # box-box contacts were exercised
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    sim.step(None, 400)
    qp, qv = sim.state()
    assert np.isfinite(qp).all() and np.isfinite(qv).all()
    assert np.all(sim.stats()["status"] == 0)
