"""Writes tests/golden/quadruped16.npz: regression fixtures of the FP64
oracle's own outputs on the seeded 16-env quadruped workload.

They are not outputs of the reference (which cannot run here) and do not
pin parity; they pin the oracle and the committed model dump against
unintended change.  Contents, env-major float64 unless noted:

  q0, v0        seeded initial state (quadruped_initial_state, keys 1000+e)
  ctrl          controls of control steps 0 and 1 (quadruped_controls)
  q1, v1, q2, v2  state after control steps 0 and 1 (4 substeps each)
  qs, vs, cs    state after 25 control steps and the controls of step 25
  ncon, nefc, niter (int32), pairs (int32, -1 padded), qacc,
  efc_type (int32, -1 padded), efc_force (0 padded)
                one substep from (qs, vs, cs)

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "mujoco-mlx-cpp_b200"), os.path.join(ROOT, "oracle")]

B, SUB, SETTLE, PAIRS, ROWS = 16, 4, 25, 32, 128


def control_step(envs, ctrl):
    for e, env in enumerate(envs):
        env.a["ctrl"][:12] = ctrl[e]
        for _ in range(SUB):
            env.step()


def one_substep(om, qs, vs, cs):
    import oracle

    out = {k: [] for k in ("ncon", "nefc", "niter", "pairs", "qacc", "efc_type", "efc_force")}
    for e in range(B):
        env = oracle.OracleEnv(om, 64, ROWS)
        env.a["qpos"][:] = qs[e]
        env.a["qvel"][:] = vs[e]
        env.a["ctrl"][:12] = cs[e]
        env.step()
        con, efc = env.contacts(), env.efc()
        pairs = np.full(PAIRS, -1, np.int32)
        pairs[:len(con)] = con[:, 13].astype(np.int32)
        et = np.full(ROWS, -1, np.int32)
        et[:env.d.nefc] = efc["type"]
        ef = np.zeros(ROWS)
        ef[:env.d.nefc] = efc["force"]
        for k, v in (("ncon", env.d.ncon), ("nefc", env.d.nefc), ("niter", env.d.niter), ("pairs", pairs), ("qacc", env.a["qacc"].copy()),
                     ("efc_type", et), ("efc_force", ef)):
            out[k].append(v)
    return {k: np.array(v, np.int32 if k in ("ncon", "nefc", "niter", "pairs", "efc_type") else np.float64) for k, v in out.items()}


def make():
    import oracle
    from mjb200 import models

    om = oracle.OracleModel(oracle.load_dump("quadruped12.dump"))
    q0, v0 = models.quadruped_initial_state(B)
    envs = [oracle.OracleEnv(om, 64, ROWS) for _ in range(B)]
    for e, env in enumerate(envs):
        env.a["qpos"][:] = q0[e]
        env.a["qvel"][:] = v0[e]
    ctrl = np.stack([models.quadruped_controls(B, k) for k in range(2)])
    res = {"q0": q0, "v0": v0, "ctrl": ctrl}
    for k in range(2):
        control_step(envs, ctrl[k])
        res[f"q{k + 1}"] = np.stack([env.a["qpos"].copy() for env in envs])
        res[f"v{k + 1}"] = np.stack([env.a["qvel"].copy() for env in envs])
    for k in range(2, SETTLE):
        control_step(envs, models.quadruped_controls(B, k))
    res["qs"] = np.stack([env.a["qpos"].copy() for env in envs])
    res["vs"] = np.stack([env.a["qvel"].copy() for env in envs])
    res["cs"] = models.quadruped_controls(B, SETTLE)
    res.update(one_substep(om, res["qs"], res["vs"], res["cs"]))
    return res


if __name__ == "__main__":
    out = os.path.join(HERE, "quadruped16.npz")
    np.savez_compressed(out, **make())
    print(out)
