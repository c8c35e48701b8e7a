"""Batched sensordata on the GPU against the FP64 oracle, after the
reference's tests/test_sensors.cpp: every step the GPU batch and the oracle
start from the same (FP32-rounded) state, so the comparison isolates the
sensor formulas from trajectory drift.

Tolerances: 1e-4 max(1, |ref|) for every sensor except the accelerometer,
whose one-step velocity difference divides FP32 velocity error by the
timestep: 3e-3 max(1, |ref|).  Quaternion sensors may differ in sign for
ballquat (framequat has w >= 0 on both sides)."""
import numpy as np
import pytest

import mjb200
import oracle

pytestmark = pytest.mark.gpu


def _run(floor, B, steps, seed, reset_at=None):
    model = mjb200.load_model_from_string(mjb200.models.sensor_xml(floor=floor))
    om = oracle.OracleModel(model.dump())
    S = model.sensors()
    q, v = mjb200.models.sensor_state(model, B, seed)
    q = q.astype(np.float32)
    v = v.astype(np.float32)
    sim = mjb200.BatchedSim(model, B)
    envs = [oracle.OracleEnv(om) for _ in range(B)]
    g = np.random.default_rng(seed)
    worst = {nm: 0.0 for nm, *_ in S}
    for t in range(steps):
        if reset_at is not None and t == reset_at:
            mask = np.zeros(B, np.int32)
            mask[::3] = 1
            sim.reset(mask)
            qr, vr = sim.state()
            for e in np.flatnonzero(mask):
                envs[e].reset_sensor_history()
            q[mask == 1] = qr[mask == 1]
            v[mask == 1] = vr[mask == 1]
        ctrl = g.uniform(-0.5, 0.5, size=(B, model.nu)).astype(np.float32)
        sim.set_state(q, v)
        sim.step(ctrl, 1)
        sd = sim.sensordata()
        qn, vn = sim.state()
        for e in range(B):
            env = envs[e]
            env.a["qpos"][:] = q[e]
            env.a["qvel"][:] = v[e]
            env.a["ctrl"][: model.nu] = ctrl[e]
            ref = env.step_sensors()
            for nm, typ, adr, dim in S:
                gv, rv = sd[e, adr: adr + dim].astype(np.float64), ref[adr: adr + dim]
                err = np.abs(gv - rv).max()
                if typ == 18:
                    err = min(err, np.abs(gv + rv).max())
                tol = (3e-3 if typ == 1 else 1e-4) * max(1.0, np.abs(rv).max())
                assert err <= tol, (t, e, nm, gv, rv)
                worst[nm] = max(worst[nm], err)
        q, v = qn, vn
    assert np.isfinite(q).all()
    return worst, S, sd


def test_sensors_free_floating_rig_match_oracle():
    worst, S, sd = _run(floor=False, B=24, steps=12, seed=3)
    print({k: "%.1e" % x for k, x in worst.items()})
    # the relative frame sensor and the touch sensor stay zero
    adr = {nm: (a, d) for nm, _, a, d in S}
    for nm in ("touch_tip", "rel_pos"):
        a, d = adr[nm]
        assert not sd[:, a: a + d].any()


def test_sensors_with_floor_contact_and_reset():
    """With the floor in reach and a masked reset halfway: reset envs read
    accelerometers without history on the next step, as in the oracle."""
    _run(floor=True, B=24, steps=10, seed=4, reset_at=5)


def test_sensordata_multi_substep_and_device_pointer():
    """step(ctrl, 4): sensordata belongs to the last substep's start state
    and its accelerometer differences against the third substep; the device
    pointer serves the same values."""
    model = mjb200.load_model_from_string(mjb200.models.sensor_xml())
    B = 8
    q, v = mjb200.models.sensor_state(model, B, 9)
    q = q.astype(np.float32)
    v = v.astype(np.float32)
    ctrl = np.full((B, model.nu), 0.2, np.float32)
    sim = mjb200.BatchedSim(model, B)
    sim.set_state(q, v)
    sim.step(ctrl, 3)
    sim.step(ctrl, 1)
    sd_a = sim.sensordata()
    b = mjb200.BatchedSim(model, B)
    b.set_state(q, v)
    b.step(ctrl, 4)
    sd_b = b.sensordata()
    assert np.array_equal(sd_a, sd_b)
    ptr, n = b.sensordata_pointer()
    b.sync()
    assert ptr and n == sd_b.size
    try:
        from cuda.bindings import runtime as rt
    except ImportError:  # older cuda-python layout
        from cuda import cudart as rt
    host = np.zeros_like(sd_b)
    err, = rt.cudaMemcpy(host.ctypes.data, ptr, host.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert int(err) == 0
    assert np.array_equal(host, sd_b)
