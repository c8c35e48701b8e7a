"""Large models: bins of free convex bodies (boxes, capsules, ellipsoids,
noisy-sphere hulls) whose per-env workspace exceeds shared memory, so the
step runs with HBM workspaces (one per resident warp).  16 bodies (nv 96)
and the bin workload's 64 bodies (nv 384, 2336 candidate pairs) against the
FP64 oracle: single steps from states visited by a GPU rollout, contact
pair lists equal (boundary flips within 1e-5 m accepted), row counts equal,
qacc relative error <= 1e-4 median and <= 5e-3 per env (the convex-pile
bound: nearly parallel curved contacts pin normals to a few 1e-4 in FP32);
rollouts stay finite without resets."""
import numpy as np
import pytest

import mjb200
import oracle
from parity import contact_sets_match, gpu_step_from, oracle_step_from, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nbody,side,B,ncon,nefc,steps", [(16, 0.5, 16, 128, 512, (40, 150)), (64, 1.0, 4, 400, 1600, (60,))])
def test_bin_parity_and_rollout(nbody, side, B, ncon, nefc, steps):
    model = mjb200.load_model_from_string(mjb200.models.bin_xml(nbody, side, seed=1))
    om = oracle.OracleModel(model.dump())
    q, v = mjb200.models.box_pile_state(model, B, seed=5)
    sim = mjb200.BatchedSim(model, B, ncon_max=ncon, nefc_max=nefc)
    shape = sim.launch_shape()
    assert shape["smem_bytes"] < 64 * 1024      # descriptors only: the workspaces are in HBM
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    done, states = 0, []
    for s in steps:
        sim.step(None, s - done)
        done = s
        states.append(sim.state())
    st = sim.stats()
    assert np.all(st["status"] == 0), st["status"]
    for qp, qv in states:
        assert np.isfinite(qp).all() and np.isfinite(qv).all()
        g = gpu_step_from(sim, qp, qv, None, ncon, nefc)
        o = oracle_step_from(om, qp.astype(np.float64), qv.astype(np.float64), np.zeros((B, 1)), ncon_max=ncon, nefc_max=nefc)
        errs = []
        for e in range(B):
            assert g["stats"]["status"][e] == 0 and o[e]["status"] == 0
            ok, nb = contact_sets_match(g["con"][e], o[e]["contacts"], g["stats"]["ncon"][e])
            assert ok, e
            if nb == 0:
                assert g["stats"]["nefc"][e] == o[e]["nefc"]
                errs.append(rel_err(g["vec"][e, 2, : om.nv], o[e]["qacc"]))
        errs = np.array(errs)
        print(nbody, "ncon", list(g["stats"]["ncon"]), "median %.2e max %.2e" % (np.median(errs), errs.max()))
        assert np.median(errs) <= 1e-4 and errs.max() <= 5e-3, (np.median(errs), errs.max())


def test_bin_workload_2048_envs_sampled_parity():
    """The bin workload at its batch size: 2048 envs of 64 free bodies,
    stepped 80 substeps from seeded poses; 64 sampled envs (every 32nd)
    checked against the oracle as above (contact pairs, row counts, qacc)."""
    model = mjb200.load_model_from_string(mjb200.models.bin_xml(64, 1.0, seed=1))
    om = oracle.OracleModel(model.dump())
    B, ncon, nefc = 2048, 400, 1600
    q, v = mjb200.models.box_pile_state(model, B, seed=7)
    sim = mjb200.BatchedSim(model, B, ncon_max=ncon, nefc_max=nefc)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    sim.step(None, 80)
    qp, qv = sim.state()
    assert np.all(sim.stats()["status"] == 0) and np.isfinite(qp).all()
    g = gpu_step_from(sim, qp, qv, None, ncon, nefc)
    idx = np.arange(0, B, 32)
    o = oracle_step_from(om, qp[idx].astype(np.float64), qv[idx].astype(np.float64), np.zeros((len(idx), 1)), ncon_max=ncon, nefc_max=nefc)
    errs, flips = [], 0
    for k, e in enumerate(idx):
        assert g["stats"]["status"][e] == 0 and o[k]["status"] == 0
        ok, nb = contact_sets_match(g["con"][e], o[k]["contacts"], g["stats"]["ncon"][e])
        assert ok, e
        flips += nb
        if nb == 0:
            assert g["stats"]["nefc"][e] == o[k]["nefc"]
            errs.append(rel_err(g["vec"][e, 2, : om.nv], o[k]["qacc"]))
    errs = np.array(errs)
    print("sampled", len(idx), "boundary flips", flips, "ncon mean", g["stats"]["ncon"][idx].mean(), "median %.2e max %.2e" % (np.median(errs), errs.max()))
    assert len(errs) >= 60
    assert np.median(errs) <= 1e-4 and errs.max() <= 5e-3, (np.median(errs), errs.max())


def test_mixed_batch_with_large_model_matches_small_model_sim(quad_model):
    """A batch mixing the quadruped with a 16-body bin runs every env with
    HBM workspaces (the bin's does not fit shared memory); the quadruped envs
    step bit-identically to a quadruped-only sim in shared memory."""
    big = mjb200.load_model_from_string(mjb200.models.bin_xml(16, 0.5, seed=1))
    Bq, Bb = 24, 8
    mixed = mjb200.BatchedSim([quad_model, big], [Bq, Bb], ncon_max=128, nefc_max=512)
    assert mixed.launch_shape()["smem_bytes"] < 64 * 1024
    small = mjb200.BatchedSim(quad_model, Bq, ncon_max=128, nefc_max=512)
    assert small.launch_shape()["smem_bytes"] > 64 * 1024
    q, v = mjb200.models.quadruped_initial_state_fast(Bq, seed=3)
    qb, vb = mjb200.models.box_pile_state(big, Bb, seed=4)
    small.set_state(q.astype(np.float32), v.astype(np.float32))
    mixed.set_state(np.concatenate([q.reshape(-1), qb.reshape(-1)]).astype(np.float32), np.concatenate([v.reshape(-1), vb.reshape(-1)]).astype(np.float32))
    for c in range(10):
        cq = mjb200.models.quadruped_controls_fast(Bq, c, seed=5).astype(np.float32)
        small.step(cq, 4)
        mixed.step(np.concatenate([cq.reshape(-1), np.zeros(0, np.float32)]), 4)
    qs, vs = small.state()
    qm, vm = mixed.state()
    nq, nv = quad_model.nq, quad_model.nv
    assert np.array_equal(qm[: Bq * nq].reshape(Bq, nq), qs) and np.array_equal(vm[: Bq * nv].reshape(Bq, nv), vs)
    assert np.isfinite(qm).all() and np.all(mixed.stats()["status"] == 0)
