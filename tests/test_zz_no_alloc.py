"""The allocation-free step (mjb200_batched_step_noalloc) against the regular
device step (mjb200_batched_step_device_ctrl) on the same inputs.

Both paths run the same stage code; only the launch mapping (persistent work
queue vs block lockstep) and the buffers differ, so after each of two calls in
a row the states must agree to max |d| <= 1e-5.  The file name keeps it last
in collection order so that it also runs after every other GPU test.
"""
import numpy as np
import pytest

import mjb200

pytestmark = pytest.mark.gpu

B = 96
NSUB = 4


def test_noalloc_matches_regular_step_twice(quad_model):
    import torch

    qpos, qvel = mjb200.models.quadruped_initial_state(B)
    qpos = qpos.astype(np.float32)
    qvel = qvel.astype(np.float32)
    ctrls = [mjb200.models.quadruped_controls(B, k).astype(np.float32) for k in range(2)]

    ref = mjb200.BatchedSim(quad_model, B)
    ref.set_state(qpos, qvel)
    sim = mjb200.BatchedSim(quad_model, B)
    dev = torch.device("cuda:0")
    qp_t = torch.from_numpy(qpos.reshape(-1).copy()).to(dev)
    qv_t = torch.from_numpy(qvel.reshape(-1).copy()).to(dev)
    warm_t = torch.zeros(qvel.size, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for k in range(2):
        ctrl_t = torch.from_numpy(ctrls[k].reshape(-1).copy()).to(dev)
        torch.cuda.synchronize()
        ref.step_device_ctrl(ctrl_t.data_ptr(), NSUB)
        ref.sync()
        rc = sim.step_noalloc(qp_t.data_ptr(), qv_t.data_ptr(), ctrl_t.data_ptr(), warm_t.data_ptr(), NSUB, stream)
        assert rc == 0, mjb200.capi.last_error()
        torch.cuda.synchronize()
        rq, rv = ref.state()
        gq = qp_t.cpu().numpy().reshape(rq.shape)
        gv = qv_t.cpu().numpy().reshape(rv.shape)
        assert np.isfinite(gq).all() and np.isfinite(gv).all()
        assert np.abs(gq - rq).max() <= 1e-5, f"call {k}: qpos differs by {np.abs(gq - rq).max():.3g}"
        assert np.abs(gv - rv).max() <= 1e-5 * max(1.0, np.abs(rv).max()), f"call {k}: qvel differs by {np.abs(gv - rv).max():.3g}"
        # the state moved: the comparison is not between two untouched copies
        assert np.abs(gq - qpos).max() > 1e-4


def test_noalloc_rejects_oversized_sim(quad_model):
    sim = mjb200.BatchedSim(quad_model, 65537)
    qp, qv, ctrl, warm = sim.device_state()
    rc = sim.step_noalloc(qp, qv, ctrl, warm, 1, sim.stream())
    assert rc == -2
    assert "65536" in mjb200.capi.last_error()
