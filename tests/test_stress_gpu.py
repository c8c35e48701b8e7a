"""Host-side ordering under stress: sims created and freed in turn, state set
from host buffers and stepped right away, mixed setters, each result checked
bitwise against a fresh sim that ran the same sequence.

Every copy that sets device state or tables is ordered on the sim's own
stream.  A blocking cudaMemcpy from pageable host memory may return before
its DMA has landed, and the sim's stream (non-blocking) is not ordered after
the legacy stream that copy runs on, so a launch right after it could read
part of the old state; likewise a zero fill on the legacy stream could land
after an upload on the sim's stream.  The largest copies (16384 envs: 1.2 MB
of qpos) give the widest window.
"""
import numpy as np
import pytest

import mjb200

pytestmark = pytest.mark.gpu


def _ctrl(B, k):
    return mjb200.models.quadruped_controls_fast(B, k, seed=8801).astype(np.float32)


def test_set_state_then_step_is_ordered(quad_model):
    """set_state followed at once by a step, 40 times on one sim and once on
    each of 8 freshly created sims: always the same bits."""
    B = 16384
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=8800)
    q, v = q.astype(np.float32), v.astype(np.float32)
    ref = mjb200.BatchedSim(quad_model, B, record=0)
    ref.set_state(q, v)
    ref.step(_ctrl(B, 0), 4)
    want = ref.state()
    warm = ref.qacc_warmstart()
    bad = 0
    for i in range(40):
        ref.set_state(q, v)
        ref.set_qacc_warmstart(np.zeros_like(warm))
        ref.step(_ctrl(B, 0), 4)
        got = ref.state()
        bad += not (np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]))
    ref.close()
    for i in range(8):
        sim = mjb200.BatchedSim(quad_model, B, record=0)
        sim.set_state(q, v)
        sim.step(_ctrl(B, 0), 4)
        got = sim.state()
        bad += not (np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]))
        sim.close()
    assert bad == 0, f"{bad} of 48 repeats differ"


def _sequence(model, B, seed):
    """A fixed sequence of setters and steps on a new sim; returns its final
    state, warm start and statistics."""
    sim = mjb200.BatchedSim(model, B)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=seed)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    sim.step(_ctrl(B, 1), 4)
    e = B // 3
    sim.set_env_state(e, q[0].astype(np.float32), np.full(model.nv, 0.1, np.float32))
    mask = np.zeros(B, np.int32)
    mask[::7] = 1
    sim.reset(mask)
    sim.step(_ctrl(B, 2), 4)
    warm = sim.qacc_warmstart()
    sim.set_qacc_warmstart(warm * 0.5)
    sim.step(_ctrl(B, 3), 2)
    sim.set_debug(8, 32)
    sim.step(_ctrl(B, 4), 1)
    out = sim.state() + (sim.qacc_warmstart(), sim.stats()["niter_sum"].copy())
    sim.close()
    return out


def test_sims_created_and_freed_with_mixed_setters(quad_model):
    """Twelve sims of different sizes created and freed in turn, each running
    the same setter sequence as a fresh sim of its size: bitwise equal."""
    sizes = [64, 1000, 4096, 777, 16384, 2368]
    ref = {B: _sequence(quad_model, B, 7000 + B) for B in sizes}
    for rep in range(2):
        for B in sizes:
            got = _sequence(quad_model, B, 7000 + B)
            for a, b in zip(got, ref[B]):
                assert np.array_equal(a, b), (rep, B)


def test_pinned_ctrl_and_state_buffers_match_pageable(quad_model):
    """Controls from a page-locked buffer go up by direct DMA (the step waits
    for that copy before returning, so the buffer may be refilled at once),
    and state(out=...) fills page-locked arrays: the results are the same
    bits as with pageable buffers, also when the pinned control buffer is
    overwritten right after each step."""
    import torch

    B = 4096
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=8810)
    q, v = q.astype(np.float32), v.astype(np.float32)
    ref = mjb200.BatchedSim(quad_model, B, record=0)
    pin = mjb200.BatchedSim(quad_model, B, record=0)
    ref.set_state(q, v)
    pin.set_state(q, v)
    cbuf = torch.empty((B, quad_model.nu), dtype=torch.float32, pin_memory=True).numpy()
    out = (torch.empty(pin.total_q, dtype=torch.float32, pin_memory=True).numpy(),
           torch.empty(pin.total_v, dtype=torch.float32, pin_memory=True).numpy())
    for k in range(6):
        c = _ctrl(B, k)
        ref.step(c.copy(), 4)
        cbuf[...] = c
        pin.step(cbuf, 4)
        cbuf[...] = np.nan   # refilled at once: the upload has already landed
        qr, vr = ref.state()
        qp, vp = pin.state(out)
        assert np.array_equal(qr, qp) and np.array_equal(vr, vp), k
    ref.close()
    pin.close()
