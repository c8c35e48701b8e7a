"""Shared helpers of the GPU parity tests: run the CUDA engine and the FP64
oracle on identical (FP32-rounded) inputs and compare."""
from __future__ import annotations

import numpy as np

import mjb200
import oracle

CONTACT_FLOATS = 16


def oracle_step_from(om, qpos, qvel, ctrl, warm=None, ncon_max=64, nefc_max=256, max_iter=0):
    """One oracle step per env from the given state; returns per-env records."""
    out = []
    for e in range(qpos.shape[0]):
        env = oracle.OracleEnv(om, ncon_max, nefc_max)
        env.a["qpos"][:] = qpos[e]
        env.a["qvel"][:] = qvel[e]
        env.a["ctrl"][: om.nu] = ctrl[e]
        if warm is not None:
            env.a["qacc_warmstart"][:] = warm[e]
        env.step(max_iter)
        out.append(dict(ncon=env.d.ncon, nefc=env.d.nefc, niter=env.d.niter, status=env.d.status,
                        contacts=env.contacts(), efc=env.efc(), qacc=env.a["qacc"].copy(),
                        qacc_smooth=env.a["qacc_smooth"].copy(), qfrc_smooth=env.a["qfrc_smooth"].copy(),
                        qfrc_constraint=env.a["qfrc_constraint"].copy(),
                        qpos=env.a["qpos"].copy(), qvel=env.a["qvel"].copy(), xpos=env.a["xpos"].copy(),
                        xquat=env.a["xquat"].copy(), subtree_com=env.a["subtree_com"].copy(), cinert=env.a["cinert"].copy(),
                        cvel=env.a["cvel"].copy(), qfrc_actuator=env.a["qfrc_actuator"].copy()))
    return out


def gpu_step_from(sim, qpos, qvel, ctrl, ncon_max=64, nefc_max=256):
    sim.set_debug(ncon_max, nefc_max)
    sim.set_state(qpos, qvel)
    sim.step(ctrl, 1)
    qp, qv = sim.state()
    con, efc, vec = sim.get_debug()
    st = sim.stats()
    return dict(qpos=qp, qvel=qv, con=con, efc=efc, vec=vec, stats=st)


def contact_sets_match(gc, oc, ncon_gpu, tol_boundary=1e-5):
    """Compare the contact lists of one env.  Returns (ok, n_boundary): a
    contact present on one side only is accepted only when its distance is
    within tol_boundary of the pair margin (round-off at the activation
    threshold); all other contacts must match pair id and order."""
    g = [(int(gc[i, 13]), float(gc[i, 12])) for i in range(ncon_gpu)]
    o = [(int(oc[i, 13]), float(oc[i, 12])) for i in range(oc.shape[0])]
    if [p for p, _ in g] == [p for p, _ in o]:
        return True, 0
    # allow boundary flips only
    gi = {p for p, _ in g}
    oi = {p for p, _ in o}
    nb = 0
    for p, dist in g + o:
        if (p in gi) != (p in oi):
            if abs(dist) > tol_boundary:
                return False, nb
            nb += 1
    return True, nb


def rel_err(a, b, floor=1.0):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), floor))
