"""The allocation-free step (mjb200_batched_step_noalloc) against the regular
device step (mjb200_batched_step_device_ctrl) on the same inputs.

The allocation-free step exists for callers that cannot have the library
allocate device memory while they step: trainers that give all free device
memory to their own caching allocator, real-time loops that cannot wait on
cudaMalloc / cudaFree, hosts with a fixed device-memory budget.  It runs the
same stage code with the sim's own launch shape, so after each of two calls
in a row the states must agree with the regular step's to max |d| <= 1e-5
(they are bitwise equal in practice).  The file name keeps it last in
collection order so that it also runs after every other GPU test.
"""
import numpy as np
import pytest

import mjb200

pytestmark = pytest.mark.gpu

NSUB = 4


def _compare_two_calls(model, qpos, qvel, ctrls):
    import torch

    B = qpos.shape[0]
    ref = mjb200.BatchedSim(model, B)
    ref.set_state(qpos, qvel)
    sim = mjb200.BatchedSim(model, B)
    dev = torch.device("cuda:0")
    qp_t = torch.from_numpy(qpos.reshape(-1).copy()).to(dev)
    qv_t = torch.from_numpy(qvel.reshape(-1).copy()).to(dev)
    warm_t = torch.zeros(qvel.size, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for k, c in enumerate(ctrls):
        ctrl_t = torch.from_numpy(c.reshape(-1).copy()).to(dev) if c is not None else None
        torch.cuda.synchronize()
        if ctrl_t is not None:
            ref.step_device_ctrl(ctrl_t.data_ptr(), NSUB)
        else:
            ref.step_device(NSUB)
        ref.sync()
        rc = sim.step_noalloc(qp_t.data_ptr(), qv_t.data_ptr(), ctrl_t.data_ptr() if ctrl_t is not None else 0, warm_t.data_ptr(), NSUB, stream)
        assert rc == 0, mjb200.capi.last_error()
        torch.cuda.synchronize()
        rq, rv = ref.state()
        gq = qp_t.cpu().numpy().reshape(rq.shape)
        gv = qv_t.cpu().numpy().reshape(rv.shape)
        assert np.isfinite(gq).all() and np.isfinite(gv).all()
        assert np.abs(gq - rq).max() <= 1e-5, f"call {k}: qpos differs by {np.abs(gq - rq).max():.3g}"
        assert np.abs(gv - rv).max() <= 1e-5 * max(1.0, np.abs(rv).max()), f"call {k}: qvel differs by {np.abs(gv - rv).max():.3g}"
        # the state moved: the comparison is not between two untouched copies
        assert np.abs(gq - qpos.reshape(gq.shape)).max() > 1e-4
    ref.close()
    sim.close()


def test_noalloc_matches_regular_step_twice(quad_model):
    B = 96
    qpos, qvel = mjb200.models.quadruped_initial_state(B)
    ctrls = [mjb200.models.quadruped_controls(B, k).astype(np.float32) for k in range(2)]
    _compare_two_calls(quad_model, qpos.astype(np.float32), qvel.astype(np.float32), ctrls)


def test_noalloc_convex_pile_matches_regular_step_twice():
    """Kernel instance with the GJK / EPA collider (mixed convex bodies)."""
    model = mjb200.load_model_from_string(mjb200.models.convex_pile_xml(6, seed=1))
    q, v = mjb200.models.box_pile_state(model, 32, seed=4)
    _compare_two_calls(model, q.astype(np.float32), v.astype(np.float32), [None, None])


def test_noalloc_replays_in_a_cuda_graph(quad_model):
    """One call outside capture (the first call on a device looks up the
    scratch address), then two calls captured into a CUDA graph on a side
    stream.  Replaying the graph on fresh inputs written into the captured
    buffers gives the regular step's state after two steps."""
    import torch

    B = 96
    dev = torch.device("cuda:0")
    qpos, qvel = mjb200.models.quadruped_initial_state(B)
    qpos, qvel = qpos.astype(np.float32), qvel.astype(np.float32)
    ctrls = [mjb200.models.quadruped_controls(B, k).astype(np.float32) for k in range(2)]
    sim = mjb200.BatchedSim(quad_model, B)
    qp_t = torch.from_numpy(qpos.reshape(-1).copy()).to(dev)
    qv_t = torch.from_numpy(qvel.reshape(-1).copy()).to(dev)
    warm_t = torch.zeros(qvel.size, dtype=torch.float32, device=dev)
    c_t = [torch.from_numpy(c.reshape(-1).copy()).to(dev) for c in ctrls]
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    assert sim.step_noalloc(qp_t.data_ptr(), qv_t.data_ptr(), c_t[0].data_ptr(), warm_t.data_ptr(), NSUB, side.cuda_stream) == 0, mjb200.capi.last_error()
    torch.cuda.synchronize()

    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        rc0 = sim.step_noalloc(qp_t.data_ptr(), qv_t.data_ptr(), c_t[0].data_ptr(), warm_t.data_ptr(), NSUB, side.cuda_stream)
        rc1 = sim.step_noalloc(qp_t.data_ptr(), qv_t.data_ptr(), c_t[1].data_ptr(), warm_t.data_ptr(), NSUB, side.cuda_stream)
    assert rc0 == 0 and rc1 == 0, mjb200.capi.last_error()

    # capture ran nothing: write the start state again, then replay
    qp_t.copy_(torch.from_numpy(qpos.reshape(-1).copy()))
    qv_t.copy_(torch.from_numpy(qvel.reshape(-1).copy()))
    warm_t.zero_()
    graph.replay()
    torch.cuda.synchronize()

    ref = mjb200.BatchedSim(quad_model, B)
    ref.set_state(qpos, qvel)
    for c in ctrls:
        ref.step(c, NSUB)
    rq, rv = ref.state()
    gq = qp_t.cpu().numpy().reshape(rq.shape)
    gv = qv_t.cpu().numpy().reshape(rv.shape)
    assert np.isfinite(gq).all() and np.isfinite(gv).all()
    assert np.abs(gq - rq).max() <= 1e-5, f"qpos differs by {np.abs(gq - rq).max():.3g}"
    assert np.abs(gv - rv).max() <= 1e-5 * max(1.0, np.abs(rv).max()), f"qvel differs by {np.abs(gv - rv).max():.3g}"
    assert np.abs(gq - qpos.reshape(gq.shape)).max() > 1e-4
    del graph
    ref.close()
    sim.close()


def test_noalloc_keeps_other_sims_launchable(quad_model):
    """A large-workspace sim, then the allocation-free step of a sim with a
    smaller workspace, then the large sim again: the shared-memory limit the
    first sim launches with must still be in place."""
    import torch

    B = 64
    big = mjb200.BatchedSim(quad_model, B)
    qpos, qvel = mjb200.models.quadruped_initial_state(B)
    ctrl = mjb200.models.quadruped_controls(B, 0).astype(np.float32)
    big.set_state(qpos.astype(np.float32), qvel.astype(np.float32))
    big.step(ctrl, NSUB)
    small_model = mjb200.load_model_from_string(mjb200.models.chain_xml(2, "free"))
    small = mjb200.BatchedSim(small_model, 8)
    assert small.launch_shape()["smem_bytes"] < big.launch_shape()["smem_bytes"]
    qp, qv, c, w = small.device_state()
    assert small.step_noalloc(qp, qv, c, w, 2, small.stream()) == 0, mjb200.capi.last_error()
    small.sync()
    big.step(ctrl, NSUB)
    q2, v2 = big.state()
    assert np.isfinite(q2).all() and np.all(big.stats()["status"] == 0)
    # the same two steps on a fresh sim give the same state
    again = mjb200.BatchedSim(quad_model, B)
    again.set_state(qpos.astype(np.float32), qvel.astype(np.float32))
    again.step(ctrl, NSUB)
    again.step(ctrl, NSUB)
    q3, v3 = again.state()
    assert np.array_equal(q2, q3) and np.array_equal(v2, v3)
    torch.cuda.synchronize()


def test_noalloc_rejects_oversized_sim(quad_model):
    sim = mjb200.BatchedSim(quad_model, 65537)
    qp, qv, ctrl, warm = sim.device_state()
    rc = sim.step_noalloc(qp, qv, ctrl, warm, 1, sim.stream())
    assert rc == -2
    assert "65536" in mjb200.capi.last_error()


def test_noalloc_rejects_hbm_workspace_model():
    """The 64-body bin needs the regular step's HBM workspace: refused with -1."""
    model = mjb200.load_model_from_string(mjb200.models.bin_xml(64, seed=0))
    sim = mjb200.BatchedSim(model, 2)
    qp, qv, ctrl, warm = sim.device_state()
    rc = sim.step_noalloc(qp, qv, ctrl, warm, 1, sim.stream())
    assert rc == -1
    assert "HBM workspace" in mjb200.capi.last_error()
