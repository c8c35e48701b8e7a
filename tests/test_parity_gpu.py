"""Single-step parity of the CUDA engine against the FP64 oracle, through the
C ABI, plus the reference's harness shapes (tests/test_gpu_vs_cpu.cpp:177-267,
tests/test_robustness.cpp:129-161): identical-env determinism, batch-size
invariance, run-to-run repeatability.

Inputs are rounded to FP32 once and fed to both sides.  Tolerances:
  * contact pair lists and constraint counts: exact, except contacts whose
    distance is within 1e-5 m of the activation threshold (round-off);
  * qacc: ||qacc_gpu - qacc_fp64|| / max(||qacc_fp64||, 1) <= 1e-4 per env and
    <= 1e-5 as the median over envs (single-step parity tests of other models
    keep their own bounds);
  * row types equal and efc_force per row within 1e-3 of max(1, max |f|);
  * one-sided boundary contacts counted, at most 1 % of the env-states;
  * qpos after one step: max |dq| <= 1e-5.
"""
import numpy as np
import pytest

import mjb200
import oracle
from parity import contact_sets_match, gpu_step_from, oracle_step_from, rel_err

pytestmark = pytest.mark.gpu

B = 64


def visited_states(om, nsteps=(0, 20, 60, 120, 240), B=B):
    """Seeded initial states and states visited by an oracle rollout with
    random position targets (resampled every 4 substeps)."""
    qpos, qvel = mjb200.models.quadruped_initial_state(B)
    ob = oracle.OracleBatch(om, B)
    ob.set_state(qpos, qvel)
    states = []
    for s in range(max(nsteps) + 1):
        if s % 4 == 0:
            ctrl = mjb200.models.quadruped_controls(B, s // 4)
            ob.set_ctrl(ctrl)
        if s in nsteps:
            qp, qv = ob.state()
            states.append((qp.astype(np.float32), qv.astype(np.float32), ctrl.astype(np.float32)))
        ob.step(1, nthread=8)
    return states


@pytest.fixture(scope="module")
def setup(quad_model):
    om = oracle.OracleModel(quad_model.dump())
    sim = mjb200.BatchedSim(quad_model, B, ncon_max=48, nefc_max=160)
    return om, sim


def test_single_step_parity(setup):
    om, sim = setup
    worst, worst_f, nbound = [], 0.0, 0
    for qp, qv, ctrl in visited_states(om):
        g = gpu_step_from(sim, qp, qv, ctrl, 48, 160)
        o = oracle_step_from(om, qp.astype(np.float64), qv.astype(np.float64), ctrl.astype(np.float64), ncon_max=48, nefc_max=160)
        errs = []
        for e in range(B):
            st = g["stats"]
            assert st["status"][e] == 0 and o[e]["status"] == 0
            ok, nb = contact_sets_match(g["con"][e], o[e]["contacts"], st["ncon"][e])
            assert ok, f"env {e}: contact sets differ"
            nbound += nb
            if nb == 0:
                assert st["ncon"][e] == o[e]["ncon"]
                assert st["nefc"][e] == o[e]["nefc"]
                n = o[e]["nefc"]
                assert list(g["efc"][e, :n, 0].astype(int)) == list(o[e]["efc"]["type"])
                f = o[e]["efc"]["force"]
                if n:
                    ferr = float(np.abs(g["efc"][e, :n, 1] - f).max()) / max(1.0, float(np.abs(f).max()))
                    assert ferr <= 1e-3, (e, ferr)
                    worst_f = max(worst_f, ferr)
                qacc_g = g["vec"][e, 2, : om.nv]
                errs.append(rel_err(qacc_g, o[e]["qacc"]))
                assert np.abs(g["qpos"][e] - o[e]["qpos"]).max() < 1e-5
        errs = np.array(errs)
        worst.append(errs.max())
        assert np.median(errs) <= 1e-5, f"median qacc rel err {np.median(errs):.3g}"
        assert errs.max() <= 1e-4, f"max qacc rel err {errs.max():.3g}"
    print("worst per-state qacc rel err:", worst, "worst efc_force err:", worst_f, "one-sided boundary contacts:", nbound)
    assert nbound <= len(worst) * B // 100


def test_smooth_quantities(setup):
    om, sim = setup
    qp, qv, ctrl = visited_states(om, nsteps=(40,))[0]
    g = gpu_step_from(sim, qp, qv, ctrl, 48, 160)
    o = oracle_step_from(om, qp.astype(np.float64), qv.astype(np.float64), ctrl.astype(np.float64))
    qas = np.stack([x["qacc_smooth"] for x in o])
    qfs = np.stack([x["qfrc_smooth"] for x in o])
    for e in range(B):
        assert rel_err(g["vec"][e, 0, : om.nv], qas[e]) < 1e-4
        assert rel_err(g["vec"][e, 1, : om.nv], qfs[e]) < 1e-5
    # recorded kinematics/dynamics getters (state at the start of the step)
    for name, key, w in (("xpos", "xpos", 3), ("xquat", "xquat", 4), ("subtree_com", "subtree_com", 3), ("cinert", "cinert", 10), ("cvel", "cvel", 6)):
        got = sim.get(name).reshape(B, -1)
        want = np.stack([x[key] for x in o])
        assert np.abs(got - want).max() < 2e-4 * max(1.0, np.abs(want).max()), name
    qfa = sim.get("qfrc_actuator").reshape(B, -1)
    assert np.abs(qfa - np.stack([x["qfrc_actuator"] for x in o])).max() < 1e-3


def test_identical_envs_bitwise(quad_model):
    sim = mjb200.BatchedSim(quad_model, 8)
    qpos, qvel = mjb200.models.quadruped_initial_state(4)
    qpos = np.concatenate([qpos, qpos]).astype(np.float32)
    qvel = np.concatenate([qvel, qvel]).astype(np.float32)
    sim.set_state(qpos, qvel)
    for s in range(40):
        c = mjb200.models.quadruped_controls(4, s // 4)
        sim.step(np.concatenate([c, c]).astype(np.float32), 1)
    qp, qv = sim.state()
    assert np.array_equal(qp[:4], qp[4:]) and np.array_equal(qv[:4], qv[4:])


def test_batch_size_invariance_and_repeatability(quad_model):
    qpos, qvel = mjb200.models.quadruped_initial_state(33)
    ctrl = mjb200.models.quadruped_controls(33, 0).astype(np.float32)
    outs = []
    for trial in range(2):
        sim = mjb200.BatchedSim(quad_model, 33)
        sim.set_state(qpos.astype(np.float32), qvel.astype(np.float32))
        sim.step(ctrl, 8)
        outs.append(sim.state())
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    one = mjb200.BatchedSim(quad_model, 1)
    one.set_state(qpos[7:8].astype(np.float32), qvel[7:8].astype(np.float32))
    one.step(ctrl[7:8], 8)
    qp1, qv1 = one.state()
    assert np.array_equal(qp1[0], outs[0][0][7]) and np.array_equal(qv1[0], outs[0][1][7])


def test_launch_variants_agree(quad_model):
    """Persistent work queue vs one-warp-per-env mapping, graph vs no graph."""
    qpos, qvel = mjb200.models.quadruped_initial_state(40)
    ctrl = mjb200.models.quadruped_controls(40, 0).astype(np.float32)
    res = []
    for kw in (dict(persistent=1, use_graph=1), dict(persistent=0, use_graph=0, warps_per_block=2)):
        sim = mjb200.BatchedSim(quad_model, 40, **kw)
        sim.set_state(qpos.astype(np.float32), qvel.astype(np.float32))
        sim.step(ctrl, 4)
        res.append(sim.state())
    assert np.array_equal(res[0][0], res[1][0])


def test_rollout_drift_1000_steps(quad_model):
    """Config-1 rollout (64 envs, 1000 substeps = 250 control steps): report the
    drift against the FP64 oracle; contact dynamics are chaotic, so only
    finiteness, no resets and a bounded trunk-height drift are asserted."""
    om = oracle.OracleModel(quad_model.dump())
    qpos, qvel = mjb200.models.quadruped_initial_state(B)
    sim = mjb200.BatchedSim(quad_model, B)
    sim.set_state(qpos.astype(np.float32), qvel.astype(np.float32))
    ob = oracle.OracleBatch(om, B)
    ob.set_state(qpos.astype(np.float32).astype(np.float64), qvel)
    drift = []
    for c in range(250):
        ctrl = mjb200.models.quadruped_controls(B, c)
        sim.step(ctrl.astype(np.float32), 4)
        ob.set_ctrl(ctrl.astype(np.float32).astype(np.float64))
        ob.step(4, nthread=8)
        if c in (0, 9, 24, 99, 249):
            qg, _ = sim.state()
            qo, _ = ob.state()
            drift.append((c + 1, float(np.abs(qg - qo).max()), float(np.median(np.abs(qg[:, 7:] - qo[:, 7:]).max(1)))))
    st = sim.stats()
    assert np.all(st["status"] == 0)
    qg, vg = sim.state()
    assert np.isfinite(qg).all() and np.isfinite(vg).all()
    print("drift (control step, max |dq|, median joint |dq|):", drift)


def test_rollout_bitwise_deterministic_across_launch_modes(quad_model):
    """2048 envs x 24 control steps give bit-identical states and iteration
    counts in lockstep (16- and 8-warp CTAs), graph-free and work-queue
    launches and on repeats."""
    B = 2048
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=777)
    ctrls = [mjb200.models.quadruped_controls_fast(B, c, seed=778).astype(np.float32) for c in range(24)]
    out = []
    for kw in (dict(), dict(), dict(use_graph=0), dict(lockstep=0), dict(warps_per_block=8)):
        sim = mjb200.BatchedSim(quad_model, B, **kw)
        sim.set_state(q.astype(np.float32), v.astype(np.float32))
        its = 0
        for c in ctrls:
            sim.step(c, 4)
            its += int(sim.stats()["niter_sum"].sum())
        qp, qv = sim.state()
        out.append((qp, qv, its))
    for qp, qv, its in out[1:]:
        assert np.array_equal(qp, out[0][0]) and np.array_equal(qv, out[0][1]) and its == out[0][2]


def test_poisoned_workspace_changes_nothing(quad_model):
    """Every shared-workspace value is written before it is read: NaN-filling
    each env's workspace before its first stage leaves the results bit-identical."""
    import subprocess
    import sys

    code = (
        "import sys, numpy as np; sys.path[:0]=%r; import mjb200\n"
        "m = mjb200.load_model_from_string(mjb200.models.quadruped_xml())\n"
        "B = 1024; q, v = mjb200.models.quadruped_initial_state_fast(B, seed=91)\n"
        "sim = mjb200.BatchedSim(m, B); sim.set_state(q.astype(np.float32), v.astype(np.float32))\n"
        "for c in range(12): sim.step(mjb200.models.quadruped_controls_fast(B, c, seed=92).astype(np.float32), 4)\n"
        "qp, qv = sim.state(); st = sim.stats()\n"
        "sys.stdout.write('%%d %%s\\n' %% (int((st['status'] != 0).sum()), hash(qp.tobytes() + qv.tobytes())))\n"
    ) % (sys.path[:3],)
    import os

    res = []
    for poison in ("0", "1"):
        env = dict(os.environ, MJB200_POISON_WORKSPACE=poison, PYTHONHASHSEED="0")
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=600)
        assert r.returncode == 0, r.stderr
        res.append(r.stdout.split())
    assert res[0][0] == "0" and res[1][0] == "0"
    assert res[0][1] == res[1][1]


def test_checkpoint_resume_bitwise(quad_model):
    """qpos, qvel and the solver's warm-start qacc checkpoint the whole step
    state: a resumed sim repeats the original run bit for bit; a caller
    warm-start equal to the converged solution needs (almost) no iterations."""
    B = 512
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=61)
    ctrls = [mjb200.models.quadruped_controls_fast(B, c, seed=62).astype(np.float32) for c in range(16)]
    a = mjb200.BatchedSim(quad_model, B)
    a.set_state(q.astype(np.float32), v.astype(np.float32))
    for c in ctrls[:8]:
        a.step(c, 4)
    qp, qv = a.state()
    warm = a.qacc_warmstart()
    b = mjb200.BatchedSim(quad_model, B)
    b.set_state(qp, qv)
    b.set_qacc_warmstart(warm)
    for c in ctrls[8:]:
        a.step(c, 4)
        b.step(c, 4)
    assert all(np.array_equal(x, y) for x, y in zip(a.state(), b.state()))
    # perfect caller warm start: the converged solution of the same step
    import torch

    b.set_state(qp, qv)
    b.set_qacc_warmstart(warm)
    b.step(ctrls[8], 1)
    it_plain = b.stats()["niter_sum"].mean()
    sol = torch.from_numpy(b.qacc_warmstart()).cuda()
    b.set_state(qp, qv)
    b.set_qacc_warmstart(warm)
    torch.cuda.synchronize()
    b.step_warmstart(sol.data_ptr(), 1)
    st = b.stats()
    assert st["niter_sum"].mean() < 0.5 * it_plain
    assert np.mean(st["warm_choice"] == 2) > 0.5


@pytest.mark.parametrize("condim", [1, 4, 6])
def test_condim_single_step_parity(condim):
    """Pyramidal contacts with condim 1 (frictionless), 4 (torsional) and 6
    (rolling): 2 (condim - 1) rows per contact (1 for condim 1), and the
    single-step qacc against the oracle within the quadruped tolerances."""
    model = mjb200.load_model_from_string(mjb200.models.quadruped_xml(condim=condim))
    om = oracle.OracleModel(model.dump())
    B = 48
    states = visited_states(om, nsteps=(30, 90), B=B)
    sim = mjb200.BatchedSim(model, B, ncon_max=48, nefc_max=320)
    rows_per = 1 if condim == 1 else 2 * (condim - 1)
    for qp, qv, ctrl in states:
        g = gpu_step_from(sim, qp, qv, ctrl, 48, 320)
        o = oracle_step_from(om, qp.astype(np.float64), qv.astype(np.float64), ctrl.astype(np.float64), ncon_max=48, nefc_max=320)
        errs = []
        for e in range(B):
            st = g["stats"]
            assert st["status"][e] == 0
            ok, nb = contact_sets_match(g["con"][e], o[e]["contacts"], st["ncon"][e])
            assert ok
            if nb == 0:
                assert st["nefc"][e] == o[e]["nefc"]
                nlim = int((o[e]["efc"]["type"] == 1).sum())
                assert o[e]["nefc"] == rows_per * o[e]["ncon"] + nlim
                errs.append(rel_err(g["vec"][e, 2, : om.nv], o[e]["qacc"]))
        errs = np.array(errs)
        assert np.median(errs) <= 1e-4 and errs.max() <= 2e-3, (condim, np.median(errs), errs.max())


def test_packed_readback_device_and_host(quad_model):
    """Packed rows (reference: mjmlx_batched_get_pack) assembled by the pack
    kernel equal the same quantities read back separately, and the device
    buffer (no host copy) holds the same rows."""
    B = 256
    sim = mjb200.BatchedSim(quad_model, B)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=71)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    for c in range(10):
        sim.step(mjb200.models.quadruped_controls_fast(B, c, seed=72).astype(np.float32), 4)
    feet = [4, 7, 10, 13]
    stride = sim.set_pack_spec(feet, 6, 12)
    assert stride == 19 + 18 + 4 + 2
    packed = sim.get_pack()
    qp, qv = sim.state()
    cf = sim.get("cfrc_ext").reshape(B, -1, 6)
    qa = sim.get("qfrc_actuator").reshape(B, -1)
    want = np.concatenate([qp, qv, np.linalg.norm(cf[:, feet, 3:], axis=2), (qa[:, 6:18] ** 2).sum(1, keepdims=True),
                           np.abs(qa[:, 6:18]).sum(1, keepdims=True)], axis=1)
    np.testing.assert_allclose(packed, want, rtol=1e-5, atol=1e-5)
    assert (packed[:, 37:41] > 0).any()          # some feet carry load
    ptr = sim.pack_device()
    sim.sync()
    assert ptr != 0
    try:
        from cuda.bindings import runtime as rt
    except ImportError:  # older cuda-python layout
        from cuda import cudart as rt
    host = np.zeros((B, stride), np.float32)
    err, = rt.cudaMemcpy(host.ctypes.data, ptr, host.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert int(err) == 0
    np.testing.assert_array_equal(host, packed)
