"""Learned warm start in per-body mode (models made only of free bodies with
nv > 64, e.g. the bin workload): one feature row and 6 outputs per body.

Checked: the layout; the feature rows against the state, converged
accelerations and contacts of the same substep read back from a twin sim
(bit-exact: the rows are copies of the same FP32 values); a net trained on
collected rows is offered to the solver (chosen by the Gauss cost for some
envs) and the step still converges to the oracle's solution (the bin
bounds: qacc median <= 1e-4, max <= 5e-3)."""
import numpy as np
import pytest

import mjb200
import oracle
from parity import contact_sets_match, rel_err

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _bin16():
    return mjb200.load_model_from_string(mjb200.models.bin_xml(16, 0.5, seed=1, condim=6, cone="elliptic"))


def _settled(model, B, seed, nsub=10):
    sim = mjb200.BatchedSim(model, B, ncon_max=128, nefc_max=768)
    q, v = mjb200.models.box_pile_state(model, B, seed=seed)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    sim.step(None, nsub)
    return sim


def test_per_body_layout_and_feature_rows():
    model = _bin16()
    d = model.dump()
    B, nb = 8, 16
    a = _settled(model, B, 3)
    b = _settled(model, B, 3)
    assert b.warmstart_layout() == (45, 6, nb)
    # a: one more substep with the contacts recorded; b: the same substep
    # inside collect, whose rows are the features written after it
    a.set_debug(128, 768)
    a.step(None, 1)
    con, _, _ = a.get_debug()
    st = a.stats()
    qp, qv = a.state()
    qacc = a.qacc_warmstart().reshape(B, -1)   # the converged qacc of that substep
    rows = B * nb
    xraw = torch.empty(rows, 45, device="cuda")
    traw = torch.empty(rows, 6, device="cuda")
    dummy = torch.zeros(1, device="cuda")
    torch.cuda.synchronize()
    assert b.warmstart_collect(dummy.data_ptr(), 1, 2, xraw.data_ptr(), traw.data_ptr(), rows) == rows
    x = xraw.cpu().numpy().reshape(B, nb, 45)
    pair = d["pair_int"].reshape(-1, 6)
    for e in range(B):
        for k in range(nb):
            body = k + 1
            q = qp[e, 7 * k: 7 * k + 7]
            row = x[e, k]
            assert row[0] == q[2] and np.array_equal(row[1:5], q[3:7])
            assert np.array_equal(row[5:11], qv[e, 6 * k: 6 * k + 6]) and np.array_equal(row[11:17], qacc[e, 6 * k: 6 * k + 6])
            want = np.zeros(28, np.float32)
            n = 0
            for c in con[e, : st["ncon"][e]]:
                b1, b2 = pair[int(c[13]), 2], pair[int(c[13]), 3]
                if body not in (b1, b2) or n == 4:
                    continue
                sg = np.float32(1.0 if b2 == body else -1.0)
                want[7 * n: 7 * n + 3] = sg * c[3:6]
                want[7 * n + 3] = c[12]
                want[7 * n + 4: 7 * n + 7] = c[0:3] - q[0:3]
                n += 1
            assert np.array_equal(row[17:], want), (e, k, row[17:], want)


def test_per_body_warm_start_is_offered_and_keeps_parity():
    model = _bin16()
    om = oracle.OracleModel(model.dump())
    B, nb, nsub = 512, 16, 24
    col = _settled(model, B, 11)
    rows = B * nb * (nsub - 1)
    xraw = torch.empty(rows, 45, device="cuda")
    traw = torch.empty(rows, 6, device="cuda")
    dummy = torch.zeros(1, device="cuda")
    torch.cuda.synchronize()
    got = col.warmstart_collect(dummy.data_ptr(), 1, nsub, xraw.data_ptr(), traw.data_ptr(), rows)
    assert got == rows
    net = mjb200.WarmStart(45, 6, seed=5)
    net.fit_normalization(xraw.data_ptr(), traw.data_ptr(), rows)
    steps, hist = net.train(xraw.data_ptr(), traw.data_ptr(), rows, epochs=4, batch=4096, lr=1e-3, seed=6)
    assert np.isfinite(hist).all() and hist[-1] < hist[0], hist
    res = {}
    for mode in ("plain", "learned"):
        sim = _settled(model, B, 21)
        if mode == "learned":
            sim.set_warmstart(net)
        it, chosen = [], []
        for c in range(6):
            sim.step(None, 4)
            st = sim.stats()
            assert np.all(st["status"] == 0)
            if c >= 1:
                it.append(st["niter_sum"] / 4.0)
                chosen.append(st["warm_choice"])
        res[mode] = (float(np.mean(it)), float(np.mean(np.array(chosen) == 2)))
        if mode == "learned":
            learned = sim
    print("bin16 mean Newton iterations per substep (plain, learned), learned choice share:", res["plain"][0], res["learned"][0], res["learned"][1])
    assert res["learned"][1] > 0.0
    # one more substep with the prediction on the table, checked against the oracle
    qp, qv = learned.state()
    learned.set_debug(128, 768)
    learned.step(None, 1)
    con, _, vec = learned.get_debug()
    st = learned.stats()
    errs = []
    for e in range(0, B, B // 16):
        env = oracle.OracleEnv(om, 128, 768)
        env.a["qpos"][:] = qp[e]
        env.a["qvel"][:] = qv[e]
        env.step()
        ok, nbd = contact_sets_match(con[e], env.contacts(), st["ncon"][e])
        assert ok
        if nbd == 0:
            assert st["nefc"][e] == env.d.nefc
            errs.append(rel_err(vec[e, 2, : om.nv], env.a["qacc"]))
    errs = np.array(errs)
    assert len(errs) >= 14 and np.median(errs) <= 1e-4 and errs.max() <= 5e-3, (np.median(errs), errs.max())
