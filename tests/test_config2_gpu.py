"""Oracle parity at the benchmarked configuration: the 12-DoF quadruped at
4096 and 16384 envs with the bench's inputs (seeded initial states, random
position targets resampled every control step), stepped with the default
launch (lockstep CTAs, persistent grid: 148 CTAs x 16 warps = 2368 envs per
wave, so 2 and 7 waves pass through the grid-stride loop), then one
recorded substep compared with the FP64 oracle on 256 sampled envs
(env = k B / 256), from the same FP32 state, controls and warm start.
Shape of the reference's harness: tests/test_gpu_vs_cpu.cpp:177-267 (CPU and
GPU backends on the same model, state and controls, per-env comparison).

Per sampled env:
  * contact pair lists equal; a contact present on one side only is allowed
    only within 1e-5 m of the activation margin, and those are counted
    (bound: at most 1 % of the sampled envs);
  * nefc and the row types equal, row by row;
  * efc_force per row within 1e-3 of max(1, max |f|) of the env;
  * qacc relative error <= 1e-4 per env and <= 1e-5 median;
  * qpos after the substep within 1e-5, qvel within 1e-4 of max(1, |qvel|);
  * cfrc_ext (contact wrench per body) within 1e-3 of max(1, max |cfrc|);
  * the packed read-back row (qpos, qvel, |foot force|, actuator-force sums,
    src/batched.cpp:1675-1727) against the same quantities from the oracle.
"""
import numpy as np
import pytest

import mjb200
import oracle
from parity import contact_sets_match, rel_err

pytestmark = pytest.mark.gpu

NSAMPLE = 256
NSUB = 4
CTRL_STEPS = 8
FEET = [4, 7, 10, 13]
NCON, NEFC = 24, 64   # the engine's automatic contact and row capacities for the quadruped, given explicitly


def _run_and_compare(model, sim, B, seed, label):
    om = oracle.OracleModel(model.dump())
    grid, warps = sim.launch_shape()["grid"], sim.launch_shape()["warps_per_block"]
    assert grid * warps < B, "the check must cover several waves of the persistent grid"
    q0, v0 = mjb200.models.quadruped_initial_state_fast(B, seed=seed)
    sim.set_state(q0.astype(np.float32), v0.astype(np.float32))
    for c in range(CTRL_STEPS):
        sim.step(mjb200.models.quadruped_controls_fast(B, c, seed=seed + 1).astype(np.float32), NSUB)
    assert np.all(sim.stats()["status"] == 0)
    qp, qv = sim.state()
    warm = sim.qacc_warmstart().reshape(B, model.nv)
    ctrl = mjb200.models.quadruped_controls_fast(B, CTRL_STEPS, seed=seed + 1).astype(np.float32)
    ncon_max, nefc_max = NCON, NEFC
    sim.set_debug(ncon_max, nefc_max)
    sim.step(ctrl, 1)
    con, efc, vec = sim.get_debug()
    st = sim.stats()
    qp1, qv1 = sim.state()
    cf = sim.get("cfrc_ext").reshape(B, -1, 6)
    stride = sim.set_pack_spec(FEET, 6, 12)
    packed = sim.get_pack()
    nboundary, qerr, ferr, cferr, niter_g, niter_o, nrows = 0, [], [], [], [], [], 0
    for k in range(NSAMPLE):
        e = k * B // NSAMPLE
        env = oracle.OracleEnv(om, ncon_max, nefc_max)
        env.a["qpos"][:] = qp[e]
        env.a["qvel"][:] = qv[e]
        env.a["ctrl"][: om.nu] = ctrl[e]
        env.a["qacc_warmstart"][:] = warm[e]
        env.step()
        assert st["status"][e] == 0 and env.d.status == 0, (e, st["status"][e], env.d.status)
        ok, nb = contact_sets_match(con[e], env.contacts(), st["ncon"][e])
        assert ok, f"env {e}: contact sets differ"
        nboundary += nb
        if nb:
            continue
        assert st["ncon"][e] == env.d.ncon and st["nefc"][e] == env.d.nefc, e
        o = env.efc()
        n = env.d.nefc
        assert list(efc[e, :n, 0].astype(int)) == list(o["type"]), e
        fscale = max(1.0, float(np.abs(o["force"]).max()) if n else 1.0)
        ferr.append(float(np.abs(efc[e, :n, 1] - o["force"]).max()) / fscale if n else 0.0)
        nrows += n
        qerr.append(rel_err(vec[e, 2, : om.nv], env.a["qacc"]))
        assert np.abs(qp1[e] - env.a["qpos"]).max() <= 1e-5, e
        assert np.abs(qv1[e] - env.a["qvel"]).max() <= 1e-4 * max(1.0, float(np.abs(env.a["qvel"]).max())), e
        ocf = env.a["cfrc_ext"].reshape(-1, 6)
        cferr.append(float(np.abs(cf[e] - ocf).max()) / max(1.0, float(np.abs(ocf).max())))
        qfa = env.a["qfrc_actuator"]
        want = np.concatenate([env.a["qpos"], env.a["qvel"], np.linalg.norm(ocf[FEET, 3:], axis=1), [(qfa[6:18] ** 2).sum(), np.abs(qfa[6:18]).sum()]])
        assert packed.shape[1] == stride
        np.testing.assert_allclose(packed[e], want, rtol=1e-3, atol=1e-3 * max(1.0, float(np.abs(want).max())))
        niter_g.append(int(st["niter_sum"][e]))
        niter_o.append(int(env.d.niter))
    qerr, ferr, cferr = np.array(qerr), np.array(ferr), np.array(cferr)
    print(f"{label}: B {B}, {len(qerr)} of {NSAMPLE} sampled envs compared, {nboundary} one-sided boundary contacts, {nrows} rows; "
          f"qacc rel err median {np.median(qerr):.2e} max {qerr.max():.2e}; efc_force err max {ferr.max():.2e}; cfrc_ext err max {cferr.max():.2e}; "
          f"Newton iterations GPU {np.mean(niter_g):.3f} oracle {np.mean(niter_o):.3f}")
    assert nboundary <= NSAMPLE // 100
    assert nrows > 0 and (st["ncon"] > 0).mean() > 0.5
    assert np.median(qerr) <= 1e-5, np.median(qerr)
    assert qerr.max() <= 1e-4, qerr.max()
    assert ferr.max() <= 1e-3, ferr.max()
    assert cferr.max() <= 1e-3, cferr.max()
    return qerr


@pytest.mark.parametrize("B", [4096, 16384])
def test_config2_sampled_parity(quad_model, B):
    sim = mjb200.BatchedSim(quad_model, B, ncon_max=NCON, nefc_max=NEFC)
    _run_and_compare(quad_model, sim, B, 9100 + B, "plain")
    sim.close()


def test_config2_learned_path_sampled_parity(quad_model):
    """The same check with the learned warm start attached (a net trained
    here on plain rollouts of 16384 envs x 4 control steps, 2 epochs): the
    prediction only moves the solver's starting point, so the converged
    solution meets the same bounds."""
    import torch

    B = 16384
    seed0 = 60000
    col = mjb200.BatchedSim(quad_model, B, record=0)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=seed0)
    col.set_state(q.astype(np.float32), v.astype(np.float32))
    nctrl = 4
    ctrl = torch.from_numpy(np.stack([mjb200.models.quadruped_controls_fast(B, c, seed=seed0 + 1) for c in range(nctrl)]).astype(np.float32)).cuda()
    width = col.warmstart_input_width()
    rows = B * NSUB * nctrl
    xraw = torch.empty(rows, width, device="cuda")
    traw = torch.empty(rows, quad_model.nv, device="cuda")
    torch.cuda.synchronize()
    got = col.warmstart_collect(ctrl.data_ptr(), nctrl, NSUB, xraw.data_ptr(), traw.data_ptr(), rows)
    net = mjb200.WarmStart(width, quad_model.nv, seed=seed0 + 2)
    net.fit_normalization(xraw.data_ptr(), traw.data_ptr(), got)
    net.train(xraw.data_ptr(), traw.data_ptr(), got, epochs=2, batch=4096, lr=1e-3, seed=seed0 + 3)
    col.close()
    sim = mjb200.BatchedSim(quad_model, B, ncon_max=NCON, nefc_max=NEFC)
    sim.set_warmstart(net)
    _run_and_compare(quad_model, sim, B, 9300, "learned")
    assert np.mean(sim.stats()["warm_choice"] == 2) > 0.1
    sim.close()
