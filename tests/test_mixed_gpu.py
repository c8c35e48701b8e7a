"""Uneven batching (the mixed-model workload): quadruped, capsule humanoid and
arm-with-gripper envs in one persistent launch, per-env mass x U[0.8, 1.2]
and friction x U[0.5, 1.25], against the FP64 oracle; and the launch-shape
autotuner, whose choice must not change any result.

Tolerances as in the quadruped parity test: contact pair lists and row
counts equal (boundary flips within 1e-5 m accepted), qacc relative error
<= 2e-3 per env and <= 1e-4 median."""
import ctypes as C

import numpy as np
import pytest

import mjb200
import oracle
from parity import contact_sets_match, rel_err

pytestmark = pytest.mark.gpu

SPLIT = (0.5, 0.3, 0.2)


def _models():
    return [mjb200.load_model_from_string(f()) for f in (mjb200.models.quadruped_xml, mjb200.models.humanoid_xml, mjb200.models.arm_xml)]


def _counts(B):
    c = [int(B * s) for s in SPLIT]
    c[0] += B - sum(c)
    return c


def _states(models, counts, seed):
    qs, vs = [], []
    for i, (m, n) in enumerate(zip(models, counts)):
        h = (0.28, 0.34) if i == 0 else (1.25, 1.35) if i == 1 else None
        q, v = mjb200.models.random_state(m, n, seed=seed + i, height=h)
        qs.append(q)
        vs.append(v)
    return qs, vs


def _ctrls(models, counts, step, seed):
    return [mjb200.models.random_controls(m, n, step, seed=seed + 10 + i) for i, (m, n) in enumerate(zip(models, counts))]


def _flat(parts):
    return np.concatenate([p.reshape(-1) for p in parts]).astype(np.float32)


def _split(flat, models, counts, attr):
    out, o = [], 0
    for m, n in zip(models, counts):
        w = getattr(m, attr)
        out.append(flat[o:o + n * w].reshape(n, w))
        o += n * w
    return out


def _randomise(sim, models, counts, rng):
    scales = []
    e0 = 0
    for m, n in zip(models, counts):
        nb = int(m.dump()["sizes"][3])
        ms = rng.uniform(0.8, 1.2, size=(n, nb))
        fs = rng.uniform(0.5, 1.25, size=n)
        assert sim.set_env_params(np.arange(e0, e0 + n), mass_scale=ms, friction_scale=fs) == 0
        scales.append((ms, fs))
        e0 += n
    return scales


def test_mixed_batch_single_step_parity():
    models = _models()
    B = 600
    counts = _counts(B)
    sim = mjb200.BatchedSim(models, counts, domain_rand=1, ncon_max=48, nefc_max=160)
    scales = _randomise(sim, models, counts, np.random.default_rng(3))
    qs, vs = _states(models, counts, 70)
    sim.set_state(_flat(qs), _flat(vs))
    for c in range(30):
        sim.step(_flat(_ctrls(models, counts, c, 70)), 4)
    assert np.all(sim.stats()["status"] == 0)
    qp, qv = sim.state()
    ctrl = _ctrls(models, counts, 30, 70)
    sim.set_debug(48, 160)
    sim.step(_flat(ctrl), 1)
    con, efc, vec = sim.get_debug()
    st = sim.stats()
    qps, qvs = _split(qp, models, counts, "nq"), _split(qv, models, counts, "nv")
    e0 = 0
    for k, (m, n) in enumerate(zip(models, counts)):
        om = oracle.OracleModel(m.dump())
        ms, fs = scales[k]
        errs, ncons = [], []
        for i in range(0, n, max(1, n // 24)):
            e = e0 + i
            env = oracle.OracleEnv(om, 48, 160)
            env.a["qpos"][:] = qps[k][i]
            env.a["qvel"][:] = qvs[k][i]
            env.a["ctrl"][: om.nu] = ctrl[k][i].astype(np.float32)
            mass = np.ascontiguousarray(ms[i].astype(np.float32), np.float64)
            rand = oracle.ORand(mass.ctypes.data_as(C.POINTER(C.c_double)), float(np.float32(fs[i])), None)
            env.step(0, rand)
            ok, nb = contact_sets_match(con[e], env.contacts(), st["ncon"][e])
            assert ok, (k, i)
            ncons.append(int(st["ncon"][e]))
            if nb == 0:
                assert st["nefc"][e] == env.d.nefc, (k, i)
                errs.append(rel_err(vec[e, 2, : om.nv], env.a["qacc"]))
        errs = np.array(errs)
        print("model", k, "contacts", ncons, "median err %.2e max %.2e" % (np.median(errs), errs.max()))
        assert np.median(errs) <= 1e-4 and errs.max() <= 2e-3, (k, np.median(errs), errs.max())
        e0 += n


def test_autotuner_choice_keeps_results():
    models = _models()
    B = 1024
    counts = _counts(B)
    qs, vs = _states(models, counts, 90)
    ctrls = [_flat(_ctrls(models, counts, c, 90)) for c in range(10)]
    out = []
    for tune in (False, True):
        sim = mjb200.BatchedSim(models, counts)
        sim.set_state(_flat(qs), _flat(vs))
        if tune:
            cands = sim.autotune(nsub=4, reps=2)
            timed = [c for c in cands if c[2] > 0]
            assert len(timed) >= 4
            best = min(timed, key=lambda c: c[2])
            shape = sim.launch_shape()
            assert shape["warps_per_block"] == best[0]
            print("autotune candidates (warps, lockstep, ms):", cands, "chosen", best)
        for c in ctrls:
            sim.step(c, 4)
        out.append(sim.state())
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_config3_8192_mixed_sampled_parity():
    """The mixed workload at its stated size: 8192 envs drawn 50/30/20 from
    the quadruped, the capsule humanoid and the arm with gripper and free
    box, mass x U[0.8, 1.2] and friction x U[0.5, 1.25] per env, in one
    persistent launch; after 8 control steps, one recorded substep compared
    with the oracle on 64 sampled envs per model (contacts, rows, qacc)."""
    models = _models()
    B = 8192
    counts = _counts(B)
    assert counts == [4097, 2457, 1638]
    sim = mjb200.BatchedSim(models, counts, domain_rand=1, ncon_max=32, nefc_max=96)
    scales = _randomise(sim, models, counts, np.random.default_rng(8192))
    qs, vs = _states(models, counts, 170)
    sim.set_state(_flat(qs), _flat(vs))
    for c in range(8):
        sim.step(_flat(_ctrls(models, counts, c, 170)), 4)
    assert np.all(sim.stats()["status"] == 0)
    qp, qv = sim.state()
    ctrl = _ctrls(models, counts, 8, 170)
    sim.set_debug(32, 96)
    sim.step(_flat(ctrl), 1)
    con, efc, vec = sim.get_debug()
    st = sim.stats()
    qps, qvs = _split(qp, models, counts, "nq"), _split(qv, models, counts, "nv")
    e0, nbound = 0, 0
    for k, (m, n) in enumerate(zip(models, counts)):
        om = oracle.OracleModel(m.dump())
        ms, fs = scales[k]
        errs, ncons = [], []
        for i in range(0, n, n // 64)[:64]:
            e = e0 + i
            env = oracle.OracleEnv(om, 32, 96)
            env.a["qpos"][:] = qps[k][i]
            env.a["qvel"][:] = qvs[k][i]
            env.a["ctrl"][: om.nu] = ctrl[k][i].astype(np.float32)
            mass = np.ascontiguousarray(ms[i].astype(np.float32), np.float64)
            rand = oracle.ORand(mass.ctypes.data_as(C.POINTER(C.c_double)), float(np.float32(fs[i])), None)
            env.step(0, rand)
            ok, nb = contact_sets_match(con[e], env.contacts(), st["ncon"][e])
            assert ok, (k, i)
            nbound += nb
            ncons.append(int(st["ncon"][e]))
            if nb == 0:
                assert st["nefc"][e] == env.d.nefc, (k, i)
                errs.append(rel_err(vec[e, 2, : om.nv], env.a["qacc"]))
        errs = np.array(errs)
        print("config 3 model", k, "envs", n, "contacts per env: mean %.1f max %d" % (np.mean(ncons), max(ncons)),
              "qacc rel err median %.2e max %.2e" % (np.median(errs), errs.max()))
        assert np.median(errs) <= 1e-4 and errs.max() <= 2e-3, (k, np.median(errs), errs.max())
        e0 += n
    assert nbound <= 3


def test_autotune_cache_reuses_choice():
    """A second sim of the same mixed batch takes the first sim's tuned
    launch shape from the cache without timing anything."""
    models = _models()
    counts = _counts(512)
    qs, vs = _states(models, counts, 95)
    a = mjb200.BatchedSim(models, counts)
    a.set_state(_flat(qs), _flat(vs))
    first = a.autotune_cached(nsub=2, reps=1)
    b = mjb200.BatchedSim(models, counts)
    b.set_state(_flat(qs), _flat(vs))
    assert b.autotune_cached(nsub=2, reps=1)
    assert b.launch_shape() == a.launch_shape()
    c = mjb200.BatchedSim(models, _counts(600))          # another batch: not cached yet
    assert not c.autotune_cached(nsub=2, reps=1) or first is False
