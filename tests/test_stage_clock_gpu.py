"""Stage clocks of the lockstep step kernel (mjb200_batched_stage_timing).

A bucket spans one stage barrier to the next: it ends when the CTA's last
warp reaches the barrier.  The quadruped's envs finish their Newton solves at
very different times (the slowest of a CTA's 16 takes about 2.4 times the
mean), and every warp waits for the slowest at the barrier after Newton, so
the Newton bucket carries that wait and the buckets after it do not.
Measured with per-warp clocks in a probe copy of the kernel: Newton about
140 K cycles per CTA-substep, collision about 39 K.  A timer that read the
clock after the barrier without waiting for the last arrival put up to 80 K
of the Newton wait into the next bucket.
"""
import numpy as np
import pytest

import mjb200

pytestmark = pytest.mark.gpu


def test_stage_buckets_keep_the_newton_wait(quad_model):
    B = 16384
    sim = mjb200.BatchedSim(quad_model, B, record=0)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=1000)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    for c in range(6):
        sim.step(mjb200.models.quadruped_controls_fast(B, c, seed=2000).astype(np.float32), 4)
    sim.sync()
    sim.stage_timing(1)
    for c in range(6, 10):
        sim.step(mjb200.models.quadruped_controls_fast(B, c, seed=2000).astype(np.float32), 4)
    t = sim.stage_timing(0)
    shape = sim.launch_shape()
    sim.close()
    ctasub = (B // shape["warps_per_block"]) * 4 * 4
    per = {k: v / ctasub for k, v in t.items() if v}
    print({k: round(x) for k, x in per.items()})
    stages = ["finish_kin", "collision", "com_crb", "rne_forces", "qacc_smooth", "constraints", "newton"]
    assert all(per.get(k, 0) > 0 for k in stages)
    assert per["newton"] == max(per[k] for k in stages)
    assert per["newton"] > 2.5 * per["collision"]
    assert per["finish_kin"] < per["newton"] / 2
