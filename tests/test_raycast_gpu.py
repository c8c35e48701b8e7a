"""Batched ray casting (mjmlx_batched_raycast) against the FP64 oracle's rays
at the same poses, for the quadruped and a mixed quadruped/humanoid/arm
batch, plus the body / group / static filters.

Tolerance: hit distance |t_gpu - t_oracle| <= 1e-4 max(1, t) (FP32 poses and
roots); geom ids equal unless two hits are within that tolerance of each
other; a miss on one side must be a miss on the other."""
import numpy as np
import pytest

import mjb200
import oracle

pytestmark = pytest.mark.gpu


def _rays(qp, nray, rng, root_xyz=True):
    B = qp.shape[0]
    centre = qp[:, None, :3] if root_xyz else np.zeros((B, 1, 3))
    pnt = centre + rng.uniform(-0.6, 0.6, size=(B, nray, 3)) + np.array([0, 0, 0.4])
    vec = rng.normal(size=(B, nray, 3))
    vec[:, : nray // 3] = [0, 0, -1]
    vec /= np.linalg.norm(vec, axis=2, keepdims=True)
    vec *= rng.uniform(0.5, 2.0, size=(B, nray, 1))
    return pnt.astype(np.float32), vec.astype(np.float32)


def _compare(om, qpos_e, pnt_e, vec_e, dist_e, gid_e, include):
    env = oracle.OracleEnv(om)
    env.a["qpos"][:] = qpos_e
    env.kinematics()
    hits = 0
    for r in range(pnt_e.shape[0]):
        t, g = env.ray(pnt_e[r].astype(np.float64), vec_e[r].astype(np.float64), include)
        tg, gg = float(dist_e[r]), int(gid_e[r])
        if t < 0 and tg < 0:
            continue
        hits += 1
        assert (t < 0) == (tg < 0), f"ray {r}: oracle {t, g} vs gpu {tg, gg}"
        assert abs(tg - t) <= 1e-4 * max(1.0, t), (r, t, tg)
        if gg != g:
            # near-tie between two geoms
            inc2 = include.copy()
            inc2[g] = 0
            t2, _ = env.ray(pnt_e[r].astype(np.float64), vec_e[r].astype(np.float64), inc2)
            assert t2 >= 0 and abs(t2 - t) <= 1e-4 * max(1.0, t), (r, g, gg, t, t2)
    return hits


def test_raycast_quadruped_matches_oracle(quad_model):
    B, nray = 64, 24
    rng = np.random.default_rng(5)
    sim = mjb200.BatchedSim(quad_model, B)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=55)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    for c in range(20):
        sim.step(mjb200.models.quadruped_controls_fast(B, c, seed=56).astype(np.float32), 4)
    qp, _ = sim.state()
    pnt, vec = _rays(qp, nray, rng)
    dist, gid = sim.raycast(pnt, vec)
    om = oracle.OracleModel(quad_model.dump())
    include = np.ones(om.ngeom, np.int32)
    hits = sum(_compare(om, qp[e].astype(np.float64), pnt[e], vec[e], dist[e], gid[e], include) for e in range(B))
    assert hits > B * nray // 3
    # filters: trunk excluded, no static geoms (the floor), no groups at all
    d2, g2 = sim.raycast(pnt, vec, bodyexclude=1)
    trunk_geoms = np.flatnonzero(quad_model.dump()["geom_bodyid"] == 1)
    assert not np.isin(g2, trunk_geoms).any()
    d3, g3 = sim.raycast(pnt, vec, flg_static=0)
    assert not (g3 == 0).any() and (g3 >= 0).any()
    d4, g4 = sim.raycast(pnt, vec, geomgroup=[0] * 6)
    assert (g4 == -1).all() and (d4 == -1).all()


def test_raycast_mixed_models_match_oracle():
    models = [mjb200.load_model_from_string(f()) for f in (mjb200.models.quadruped_xml, mjb200.models.humanoid_xml, mjb200.models.arm_xml)]
    counts = [24, 16, 16]
    sim = mjb200.BatchedSim(models, counts)
    qs, vs = [], []
    for i, (m, n) in enumerate(zip(models, counts)):
        h = (0.28, 0.34) if i == 0 else (1.25, 1.35) if i == 1 else None
        q, v = mjb200.models.random_state(m, n, seed=80 + i, height=h)
        qs.append(q)
        vs.append(v)
    sim.set_state(np.concatenate([q.reshape(-1) for q in qs]).astype(np.float32), np.concatenate([v.reshape(-1) for v in vs]).astype(np.float32))
    qp, _ = sim.state()
    rng = np.random.default_rng(8)
    B, nray = sum(counts), 16
    # per-env root position for ray origins (the arm has no free root: origin near the table)
    roots = np.zeros((B, 3))
    o = 0
    e = 0
    for m, n in zip(models, counts):
        for i in range(n):
            roots[e] = qp[o + m.nq * i: o + m.nq * i + 3] if m.nq != 16 else [0.3, 0.0, 0.2]
            e += 1
        o += m.nq * n
    pnt, vec = _rays(np.concatenate([roots, np.zeros((B, 4))], axis=1), nray, rng)
    dist, gid = sim.raycast(pnt, vec)
    e, o, hits = 0, 0, 0
    for m, n in zip(models, counts):
        om = oracle.OracleModel(m.dump())
        include = np.ones(om.ngeom, np.int32)
        for i in range(n):
            hits += _compare(om, qp[o + m.nq * i: o + m.nq * (i + 1)].astype(np.float64), pnt[e], vec[e], dist[e], gid[e], include)
            e += 1
        o += m.nq * n
    assert hits > B * nray // 4


def test_raycast_with_16_warp_ctas(quad_model):
    """The geom-pose pass runs with the sim's launch shape, including the
    largest lockstep CTA (16 warps)."""
    B = 48
    sim = mjb200.BatchedSim(quad_model, B, warps_per_block=16)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=57)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    rng = np.random.default_rng(3)
    pnt, vec = _rays(q, 8, rng)
    dist, gid = sim.raycast(pnt, vec)
    ref = mjb200.BatchedSim(quad_model, B)
    ref.set_state(q.astype(np.float32), v.astype(np.float32))
    d2, g2 = ref.raycast(pnt, vec)
    assert np.array_equal(gid, g2) and np.array_equal(dist, d2)
