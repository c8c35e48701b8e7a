"""Learned warm start on the GPU: the tcgen05 GEMM against torch, the
network's forward pass and gradients against the CPU reference
(oracle/mlp_ref.py), training, and what the trained network gains over the
plain solver on the quadruped.

Tolerances: GEMM max error <= 1e-5 of max |C| (bf16 products are exact in
FP32, only the summation order differs); forward / gradients against the
bf16-mirrored reference <= 2e-2 relative (Frobenius, per parameter block)
and against the exact float64 network <= 6e-2 (bf16 rounding of
activations and weights).
"""
import numpy as np
import pytest

import mjb200
import mlp_ref
import oracle
from parity import contact_sets_match, rel_err

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (300, 256, 192), (1000, 64, 256), (64, 192, 4096), (256, 128, 128), (130, 512, 256)])
def test_gemm_matches_torch(M, N, K):
    g = torch.Generator().manual_seed(M * 7919 + N * 31 + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    C = torch.full((M, N), float("nan"), device="cuda")
    torch.cuda.synchronize()
    assert mjb200.gemm_bf16(A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K) == 0, mjb200.capi.last_error()
    torch.cuda.synchronize()
    ref = A.double() @ B.double().T
    err = (C.double() - ref).abs().max().item() / ref.abs().max().item()
    assert err <= 1e-5, err


def _net_and_data(n, seed=0, in_raw=129, nout=18, out_scale=1.0):
    rng = np.random.default_rng(seed)
    net = mjb200.WarmStart(in_raw, nout, seed=seed + 11)
    p = net.get_params()
    if out_scale != 1.0:
        layers = mlp_ref.unpack(p, net.in_pad)
        W3, b3 = layers[3]
        layers[3] = (W3 * out_scale, b3)
        p = mlp_ref.pack(layers).astype(np.float32)
        net.set_params(p)
    xraw = (rng.normal(size=(n, in_raw)) * rng.uniform(0.1, 3, size=in_raw) + rng.normal(size=in_raw)).astype(np.float32)
    traw = (rng.normal(size=(n, nout)) * 2 + 0.5).astype(np.float32)
    im, is_ = xraw.mean(0), xraw.std(0)
    om, os_ = traw.mean(0), traw.std(0)
    net.set_normalization(im, is_, om, os_)
    return net, p, xraw, traw, (im, is_, om, os_)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_matches_cpu_reference():
    n = 200
    net, p, xraw, traw, (im, is_, om, os_) = _net_and_data(n, seed=1, out_scale=10.0)
    x = torch.from_numpy(xraw).cuda()
    y = torch.empty(n, net.nout, device="cuda")
    torch.cuda.synchronize()
    net.forward(x.data_ptr(), n, y.data_ptr())
    got = y.cpu().numpy()
    ref = mlp_ref.forward(p, xraw, im, is_, net.in_pad)[:, : net.nout]
    exact = mlp_ref.forward(p, xraw, im, is_, net.in_pad, bf16=False)[:, : net.nout]
    assert _rel(got, ref) <= 2e-2
    assert _rel(got, exact) <= 6e-2


@pytest.mark.parametrize("n", [256, 4096])
def test_gradients_match_cpu_reference(n):
    """n = 4096 runs the weight-gradient GEMMs with K split over 16 CTAs per
    output tile (64 K chunks) and the ordered reduction of the partials."""
    net, p, xraw, traw, (im, is_, om, os_) = _net_and_data(n, seed=2, out_scale=10.0)
    x = torch.from_numpy(xraw).cuda()
    t = torch.from_numpy(traw).cuda()
    torch.cuda.synchronize()
    loss, g = net.gradients(x.data_ptr(), t.data_ptr(), n)
    lref, gref = mlp_ref.loss_and_grads(p, xraw, traw, im, is_, om, os_, net.in_pad, net.nout)
    lex, gex = mlp_ref.loss_and_grads(p, xraw, traw, im, is_, om, os_, net.in_pad, net.nout, bf16=False)
    assert loss == pytest.approx(lref, rel=1e-2)
    o = 0
    for r, c in mlp_ref.layer_shapes(net.in_pad):
        for size in (r * c, r):
            blk = slice(o, o + size)
            assert _rel(g[blk], gref[blk]) <= 2e-2, (r, c, size, _rel(g[blk], gref[blk]))
            assert _rel(g[blk], gex[blk]) <= 6e-2, (r, c, size, _rel(g[blk], gex[blk]))
            o += size
    assert o == net.nparams


def test_training_fits_a_smooth_map():
    n, in_raw, nout = 65536, 129, 18
    rng = np.random.default_rng(3)
    xraw = rng.normal(size=(n, in_raw)).astype(np.float32)
    A = rng.normal(size=(in_raw, nout)) / np.sqrt(in_raw)
    traw = np.tanh(xraw @ A * 2).astype(np.float32)
    net = mjb200.WarmStart(in_raw, nout, seed=4)
    x = torch.from_numpy(xraw).cuda()
    t = torch.from_numpy(traw).cuda()
    torch.cuda.synchronize()
    net.fit_normalization(x.data_ptr(), t.data_ptr(), n)
    steps, hist = net.train(x.data_ptr(), t.data_ptr(), n, epochs=8, batch=2048, lr=2e-3, seed=5)
    assert steps == 8 * (n // 2048)
    assert np.isfinite(hist).all()
    assert hist[-1] < 0.25 * hist[0], hist


def _collect_and_train(model, B, nctrl, epochs, seed0=50000):
    sim = mjb200.BatchedSim(model, B)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=seed0)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    ctrl = np.stack([mjb200.models.quadruped_controls_fast(B, c, seed=seed0 + 1) for c in range(nctrl)]).astype(np.float32)
    ctrl_d = torch.from_numpy(ctrl).cuda()
    width = sim.warmstart_input_width()
    rows = B * nctrl * 4
    xraw = torch.empty(rows, width, device="cuda")
    traw = torch.empty(rows, model.nv, device="cuda")
    torch.cuda.synchronize()
    got = sim.warmstart_collect(ctrl_d.data_ptr(), nctrl, 4, xraw.data_ptr(), traw.data_ptr(), rows)
    assert got == rows
    net = mjb200.WarmStart(width, model.nv, seed=7)
    net.fit_normalization(xraw.data_ptr(), traw.data_ptr(), rows)
    steps, hist = net.train(xraw.data_ptr(), traw.data_ptr(), rows, epochs=epochs, batch=4096, lr=1e-3, seed=8)
    return net, hist


@pytest.fixture(scope="module")
def trained_quad_net(quad_model):
    net, hist = _collect_and_train(quad_model, 2048, 64, 6)
    return net, hist


def test_trained_net_cuts_newton_iterations(quad_model, trained_quad_net):
    """Same initial states and controls, plain vs learned warm start: the
    learned path must need fewer Newton iterations per substep on average."""
    net, hist = trained_quad_net
    assert hist[-1] < hist[0]
    B, nctrl = 2048, 24
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=777)
    ctrl = [mjb200.models.quadruped_controls_fast(B, c, seed=778).astype(np.float32) for c in range(nctrl)]
    res = {}
    for mode in ("plain", "learned"):
        sim = mjb200.BatchedSim(quad_model, B)
        if mode == "learned":
            sim.set_warmstart(net)
        sim.set_state(q.astype(np.float32), v.astype(np.float32))
        it, chosen = [], []
        for c in range(nctrl):
            sim.step(ctrl[c], 4)
            st = sim.stats()
            assert np.all(st["status"] == 0)
            if c >= 2:
                it.append(st["niter_sum"] / 4.0)
                chosen.append(st["warm_choice"])
        res[mode] = (float(np.mean(it)), float(np.mean(np.array(chosen) == 2)))
    print("mean Newton iterations per substep (plain, learned), learned choice share:", res["plain"][0], res["learned"][0], res["learned"][1])
    assert res["learned"][1] > 0.2
    assert res["learned"][0] < res["plain"][0]


def test_learned_path_single_step_parity(quad_model, trained_quad_net):
    """With a prediction on the table, the solver still converges to the
    oracle's solution (same tolerances as the plain parity test)."""
    net, _ = trained_quad_net
    B = 2048
    om = oracle.OracleModel(quad_model.dump())
    sim = mjb200.BatchedSim(quad_model, B, ncon_max=48, nefc_max=160)
    sim.set_warmstart(net)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=4242)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    c0 = mjb200.models.quadruped_controls_fast(B, 0, seed=4243).astype(np.float32)
    sim.step(c0, 7)                      # features of the last substep are now valid
    qp, qv = sim.state()
    sim.set_debug(48, 160)
    sim.step(c0, 1)
    con, efc, vec = sim.get_debug()
    st = sim.stats()
    qa_gpu = vec
    sample = range(0, B, B // 64)
    errs = []
    for e in sample:
        env = oracle.OracleEnv(om, 48, 160)
        env.a["qpos"][:] = qp[e]
        env.a["qvel"][:] = qv[e]
        env.a["ctrl"][: om.nu] = c0[e]
        env.step()
        ok, nb = contact_sets_match(con[e], env.contacts(), st["ncon"][e])
        assert ok
        if nb == 0:
            assert st["nefc"][e] == env.d.nefc
            errs.append(rel_err(qa_gpu[e, 2, : om.nv], env.a["qacc"]))
            if errs[-1] > 1e-3:
                print("env", e, "err", errs[-1], "status", st["status"][e], env.d.status, "niter", st["niter_sum"][e], env.d.niter, "choice",
                      st["warm_choice"][e], "ncon", st["ncon"][e], "qacc_smooth err", rel_err(qa_gpu[e, 0, : om.nv], env.a["qacc_smooth"]),
                      "qfrc_smooth err", rel_err(qa_gpu[e, 1, : om.nv], env.a["qfrc_smooth"]))
    errs = np.array(errs)
    assert np.median(errs) <= 1e-4 and errs.max() <= 2e-3, (np.median(errs), errs.max())
    assert np.mean(st["warm_choice"] == 2) > 0.2


@pytest.mark.parametrize("B", [128, 1000, 16384])
def test_fused_inference_matches_unfused(B):
    """The fused inference kernel (gather + 4 layers in one launch) against
    the gather kernel + 4 GEMMs: same bf16 rounding points, FP32 sums in a
    different order, so agreement to 1e-3 of the prediction's scale."""
    net, p, xraw, traw, (im, is_, om, os_) = _net_and_data(256, seed=9, out_scale=10.0)
    rng = np.random.default_rng(10)
    nfeat, nu = 117, 12
    feat = torch.from_numpy((rng.normal(size=(B, 120)) * 2).astype(np.float32)).cuda()
    ctrl = torch.from_numpy(rng.normal(size=(B, nu)).astype(np.float32)).cuda()
    prev = torch.from_numpy(rng.normal(size=(B, 18)).astype(np.float32)).cuda()
    outs = []
    for fused in (True, False):
        pred = torch.full((B, 18), float("nan"), device="cuda")
        torch.cuda.synchronize()
        net.predict(feat.data_ptr(), 120, nfeat, ctrl.data_ptr(), nu, prev.data_ptr(), pred.data_ptr(), B, fused)
        outs.append(pred.cpu().numpy())
    assert np.isfinite(outs[0]).all()
    scale = np.abs(outs[1] - prev.cpu().numpy()).max()
    assert np.abs(outs[0] - outs[1]).max() <= 1e-3 * scale + 1e-6, np.abs(outs[0] - outs[1]).max() / scale


def test_gemm_bounded_wait_gives_up_and_context_survives():
    """Every mbarrier / flag wait of the tcgen05 GEMM is bounded.  A gate
    word that nothing sets makes the first MMA's wait run out (limit 50 ms):
    the kernel returns with the error word set and C untouched, and the next
    GEMM on the same context is correct.  With the gate open the gated GEMM
    gives the plain result."""
    import time

    M, N, K = 300, 256, 512
    g = torch.Generator().manual_seed(5)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    C = torch.full((M, N), float("nan"), device="cuda")
    gate = torch.zeros(1, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = mjb200.capi.lib.mjb200_gemm_bf16_gated(A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, gate.data_ptr(), 0.05, err.data_ptr(), None)
    assert rc == 0, mjb200.capi.last_error()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    assert int(err.item()) == 1
    assert torch.isnan(C).all()
    assert dt < 5.0
    ref = (A.double() @ B.double().T)
    C2 = torch.full((M, N), float("nan"), device="cuda")
    assert mjb200.gemm_bf16(A.data_ptr(), B.data_ptr(), C2.data_ptr(), M, N, K) == 0
    torch.cuda.synchronize()
    assert (C2.double() - ref).abs().max().item() <= 1e-5 * ref.abs().max().item()
    gate.fill_(1)
    err.zero_()
    C3 = torch.full((M, N), float("nan"), device="cuda")
    torch.cuda.synchronize()
    assert mjb200.capi.lib.mjb200_gemm_bf16_gated(A.data_ptr(), B.data_ptr(), C3.data_ptr(), M, N, K, gate.data_ptr(), 0.5, err.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(C3, C2)


def test_fused_kernel_inference_matches_tcgen05_inference(quad_model, trained_quad_net):
    """The step kernel's own inference (bf16 mma.sync tiles shared by the
    CTA's warps) against the net's tcgen05 inference on the features the
    kernel captured: same bf16 rounding points, FP32 sums in another order,
    so agreement to 1e-3 of the prediction's scale.  1003 envs leave a last
    CTA with 3 valid warps, whose rows must not disturb the others."""
    net, _ = trained_quad_net
    B = 1003
    sim = mjb200.BatchedSim(quad_model, B)
    sim.set_warmstart(net)
    q, v = mjb200.models.quadruped_initial_state_fast(B, seed=5150)
    sim.set_state(q.astype(np.float32), v.astype(np.float32))
    for c in range(3):
        sim.step(mjb200.models.quadruped_controls_fast(B, c, seed=5151).astype(np.float32), 4)
    sim.set_debug(24, 64)
    sim.step(mjb200.models.quadruped_controls_fast(B, 3, seed=5151).astype(np.float32), 4)
    feat, pred = sim.warmstart_debug()
    nv = quad_model.nv
    pred = pred.reshape(B, nv)
    nqf = quad_model.nq - 2
    prev = np.ascontiguousarray(feat[:, nqf + 2 * nv: nqf + 3 * nv])
    assert np.isfinite(feat).all() and np.isfinite(pred).all()
    f_d = torch.from_numpy(feat).cuda()
    p_d = torch.from_numpy(prev).cuda()
    out = torch.full((B, nv), float("nan"), device="cuda")
    torch.cuda.synchronize()
    net.predict(f_d.data_ptr(), feat.shape[1], feat.shape[1], 0, 0, p_d.data_ptr(), out.data_ptr(), B, True)
    ref = out.cpu().numpy()
    scale = np.abs(ref - prev).max()
    err = np.abs(pred - ref).max()
    print("fused in-kernel vs tcgen05 prediction: max diff %.3g, scale %.3g" % (err, scale))
    assert scale > 0 and err <= 1e-3 * scale + 1e-6
    st = sim.stats()
    assert np.all(st["status"] == 0)
    assert np.mean(st["warm_choice"] == 2) > 0.1
