"""Small fixed workloads for profiling the engine's kernels under a profiler
(e.g. ncu with -k / -c), one process, one GPU.

    python -m mjb200.profile_driver step    --envs 4096 --ctrl 3
    python -m mjb200.profile_driver learned --envs 4096 --ctrl 3
    python -m mjb200.profile_driver gemm    --rows 16384
    python -m mjb200.profile_driver sensitivity --envs 4096
    python -m mjb200.profile_driver aux --envs 16384

`step`: the quadruped workload (4 substeps per control step, seeded random
position targets) on the plain solver; `learned`: the same after a short
warm-start training (collect + 2 epochs) with the net attached; `gemm`: the
MLP's forward GEMM shapes (rows x 192 -> 256 -> 256 -> 256 -> 64) and one
weight-gradient shape (256 x 256, K = 4096), each launched `--repeat` times;
`aux`: the small kernels (pack, reset, geom poses and rays, the training
kernels around the GEMMs) at sizes above L2;
`sensitivity`: Newton iterations of one substep from warm starts at known
distances from the converged solution x* (x* + eps (previous - x*)), which
bounds what any predicted warm start can save.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def _quick_warmstart(mjb200, torch, m, B, nctrl=8, epochs=2, seed=50000):
    """Warm-start net trained briefly on plain rollouts of the same model."""
    col = mjb200.BatchedSim(m, B, record=0)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=seed)
    col.set_state(q.astype(np.float32), v.astype(np.float32))
    ctrl = torch.from_numpy(np.stack([mjb200.models.quadruped_controls_fast(B, c, seed=seed + 1) for c in range(nctrl)]).astype(np.float32)).cuda()
    width = col.warmstart_input_width()
    rows = B * 4 * nctrl
    x = torch.empty(rows, width, device="cuda")
    t = torch.empty(rows, m.nv, device="cuda")
    torch.cuda.synchronize()
    n = col.warmstart_collect(ctrl.data_ptr(), nctrl, 4, x.data_ptr(), t.data_ptr(), rows)
    net = mjb200.WarmStart(width, m.nv, seed=seed + 2)
    net.fit_normalization(x.data_ptr(), t.data_ptr(), n)
    net.train(x.data_ptr(), t.data_ptr(), n, epochs=epochs, batch=4096, lr=1e-3, seed=seed + 3)
    col.close()
    return net


def _sensitivity(mjb200, m, B):
    nv = m.nv
    sim = mjb200.BatchedSim(m, B, record=0)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=31)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    for c in range(10):
        sim.step(mjb200.models.quadruped_controls_fast(B, c, seed=32).astype(np.float32), 4)
    ctrl = mjb200.models.quadruped_controls_fast(B, 10, seed=32).astype(np.float32)
    sim.step(ctrl, 3)
    sq, sv = sim.state()
    prev = sim.qacc_warmstart().reshape(B, nv)

    def run(cand):
        sim.set_state(sq, sv)
        sim.set_qacc_warmstart(cand.astype(np.float32))
        sim.step(ctrl, 1)
        st = sim.stats()
        return st["niter_sum"].copy(), st["nefc"].copy(), sim.qacc_warmstart().reshape(B, nv)

    it0, nefc, xs = run(prev)
    print("envs %d, with contacts %d" % (B, int((nefc > 0).sum())))
    print("warm start                      mean iterations")
    print("previous qacc                   %.3f" % it0.mean())
    for eps in (0.0, 1e-3, 1e-2, 3e-2, 0.1, 0.3, 0.6):
        it, _, _ = run(xs + eps * (prev - xs))
        print("x* + %-5g (prev - x*)         %.3f" % (eps, it.mean()))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["step", "learned", "gemm", "sensitivity", "bin", "convex", "aux"])
    ap.add_argument("--envs", type=int, default=4096)
    ap.add_argument("--ctrl", type=int, default=3, help="control steps (4 substeps each)")
    ap.add_argument("--rows", type=int, default=16384)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--cone", default="pyramidal", choices=["pyramidal", "elliptic"], help="bin / convex: friction cone")
    ap.add_argument("--condim", type=int, default=3, help="bin / convex: contact dimensionality")
    ap.add_argument("--time", action="store_true", help="bin / convex: time the control steps with CUDA events")
    ap.add_argument("--learned", action="store_true", help="bin --time: also train the per-body warm start and time it")
    ap.add_argument("--stages", action="store_true", help="bin --time: per-stage share of the warps' cycles over one control step")
    ap.add_argument("--train-substeps", type=int, default=24, help="bin --learned: substeps of the collection rollout")
    ap.add_argument("--train-epochs", type=int, default=8)
    a = ap.parse_args(argv)

    import torch

    import mjb200

    if a.what == "gemm":
        g = torch.Generator().manual_seed(0)
        shapes = [(a.rows, 256, 192), (a.rows, 256, 256), (a.rows, 64, 256), (256, 256, 4096)]
        for M, N, K in shapes:
            A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
            B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
            C = torch.empty(M, N, device="cuda")
            torch.cuda.synchronize()
            for _ in range(a.repeat):
                if mjb200.gemm_bf16(A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K) != 0:
                    raise RuntimeError(mjb200.capi.last_error())
            torch.cuda.synchronize()
        print("gemm done")
        return

    if a.what == "aux":
        # the engine's small kernels, each a few times at sizes above L2
        # where the kernel scales: packed read-back (16384 envs), masked
        # reset (16384 envs), geom poses + ray casts (4096 envs x 64 rays),
        # and the training kernels (feature gather, column statistics, bias
        # gradient sums, Adam) on 262144 rows of 129 inputs
        m = mjb200.load_model_from_string(mjb200.models.quadruped_xml())
        B = a.envs
        sim = mjb200.BatchedSim(m, B)
        q, v = mjb200.models.quadruped_initial_state_fast(B, seed=1000)
        sim.set_state(q.astype(np.float32), v.astype(np.float32))
        sim.step(mjb200.models.quadruped_controls_fast(B, 0, seed=2000).astype(np.float32), 4)
        sim.set_pack_spec([4, 7, 10, 13], 6, 12)
        for _ in range(a.repeat):
            sim.pack_device()
        sim.sync()
        for _ in range(a.repeat):
            sim.reset(np.ones(B, np.int32))
        nb = min(B, 4096)
        rs = mjb200.BatchedSim(m, nb)
        g = np.random.default_rng(0)
        pnt = np.zeros((nb, 64, 3), np.float32)
        pnt[:, :, 2] = 1.0
        pnt[:, :, :2] = g.uniform(-0.4, 0.4, size=(nb, 64, 2))
        vec = np.zeros((nb, 64, 3), np.float32)
        vec[:, :, 2] = -1.0
        for _ in range(a.repeat):
            rs.raycast(pnt, vec)
        rows, width = 262144, 129
        x = torch.randn(rows, width, device="cuda")
        t = torch.randn(rows, m.nv, device="cuda")
        net = mjb200.WarmStart(width, m.nv, seed=3)
        torch.cuda.synchronize()
        net.fit_normalization(x.data_ptr(), t.data_ptr(), rows)
        net.train(x.data_ptr(), t.data_ptr(), rows, epochs=1, batch=4096, lr=1e-3, seed=4)
        torch.cuda.synchronize()
        print("aux done")
        return

    if a.what in ("bin", "convex"):
        # large-model path (HBM workspaces, row-sparse H, zero-skipping
        # Cholesky) on the 64-body bin, or the GJK / EPA kernel instance on
        # the 6-body convex pile; a.ctrl substeps after 20 settling substeps
        # (--time: a.ctrl control steps of 4 substeps, CUDA events around
        # each, Newton iterations per substep from the step statistics)
        if a.what == "bin":
            xml = mjb200.models.bin_xml(64, 1.0, seed=1, condim=a.condim, cone=a.cone)
        else:
            xml = mjb200.models.convex_pile_xml(6, seed=1, condim=a.condim, cone=a.cone)
        m = mjb200.load_model_from_string(xml)
        rows = a.condim if (a.cone == "elliptic" and a.condim > 1) else max(1, 2 * (a.condim - 1))
        ncon = 400 if a.what == "bin" else 40
        sim = mjb200.BatchedSim(m, a.envs, record=0, ncon_max=ncon, nefc_max=ncon * rows)
        q, v = mjb200.models.box_pile_state(m, a.envs, seed=5)
        sim.set_state(q.astype(np.float32), v.astype(np.float32))
        sim.step(None, 20)
        if not a.time:
            for c in range(a.ctrl):
                sim.step(None, 1)
            sim.sync()
            st = sim.stats()
            print(a.what, "done: shape", sim.launch_shape(), "ncon mean", st["ncon"].mean(), "nefc mean", st["nefc"].mean(), "status", np.unique(st["status"]))
            return
        sim.sync()
        net = None
        if a.learned:
            # per-body warm start trained on a rollout from other seeded poses
            col = mjb200.BatchedSim(m, a.envs, record=0, ncon_max=ncon, nefc_max=ncon * rows)
            qc, vc = mjb200.models.box_pile_state(m, a.envs, seed=905)
            col.set_state(qc.astype(np.float32), vc.astype(np.float32))
            col.step(None, 20)
            in_raw, nout, rpe = col.warmstart_layout()
            n = a.envs * rpe * (a.train_substeps - 1)
            x = torch.empty(n, in_raw, device="cuda")
            t = torch.empty(n, nout, device="cuda")
            dummy = torch.zeros(1, device="cuda")
            torch.cuda.synchronize()
            got = col.warmstart_collect(dummy.data_ptr(), 1, a.train_substeps, x.data_ptr(), t.data_ptr(), n)
            net = mjb200.WarmStart(in_raw, nout, seed=906)
            net.fit_normalization(x.data_ptr(), t.data_ptr(), got)
            _, hist = net.train(x.data_ptr(), t.data_ptr(), got, epochs=a.train_epochs, batch=4096, lr=1e-3, seed=907)
            print(json.dumps(dict(train_rows=got, layout=[in_raw, nout, rpe], epoch_loss=[float(h) for h in hist])))
            del x, t
            col.close()
        modes = ("plain", "learned") if a.learned else ("plain",)
        for mode in modes:
            s2 = sim if mode == "plain" else mjb200.BatchedSim(m, a.envs, record=0, ncon_max=ncon, nefc_max=ncon * rows)
            if mode == "learned":
                s2.set_warmstart(net)
                s2.set_state(q.astype(np.float32), v.astype(np.float32))
                s2.step(None, 20)
                s2.sync()
            else:
                s2.set_state(q.astype(np.float32), v.astype(np.float32))
                s2.step(None, 20)
                s2.sync()
            stream = torch.cuda.ExternalStream(s2.stream())   # the sim launches on its own stream
            ms, its, itmax, chosen = [], [], [], []
            for c in range(a.ctrl):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                s2.step(None, 4)
                e1.record(stream)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
                st = s2.stats()
                its.append(st["niter_sum"] / 4.0)
                itmax.append(st["niter_max"])
                chosen.append(st["warm_choice"])
            its = np.concatenate(its)
            out = dict(workload=f"{a.what} {a.cone} condim {a.condim}", mode=mode, envs=a.envs, ms_per_control_step=float(np.median(ms)),
                       env_steps_per_s=a.envs * 1e3 / float(np.median(ms)), newton_iter_mean=float(its.mean()),
                       newton_iter_p99=float(np.percentile(its, 99)), newton_iter_max=int(np.max(itmax)),
                       learned_choice_share=float(np.mean(np.concatenate(chosen) == 2)), ncon_mean=float(st["ncon"].mean()),
                       nefc_mean=float(st["nefc"].mean()), status=[int(x) for x in np.unique(st["status"])], shape=s2.launch_shape())
            print(json.dumps(out))
            if a.stages and mode == "plain":
                s2.stage_timing(1)
                s2.step(None, 4)
                cyc = s2.stage_timing(0)
                tot = sum(cyc.values()) or 1
                print(json.dumps({k: round(v / tot, 4) for k, v in cyc.items() if v}))
        return

    m = mjb200.load_model_from_string(mjb200.models.quadruped_xml())
    B = a.envs
    if a.what == "sensitivity":
        _sensitivity(mjb200, m, B)
        return
    sim = mjb200.BatchedSim(m, B, record=0)
    if a.what == "learned":
        net = _quick_warmstart(mjb200, torch, m, B)
        sim.set_warmstart(net)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=1000)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    for c in range(a.ctrl):
        sim.step(mjb200.models.quadruped_controls_fast(B, c, seed=2000).astype(np.float32), 4)
    sim.sync()
    print("step done", sim.stats()["niter_sum"].mean() / 4.0)


if __name__ == "__main__":
    main()
