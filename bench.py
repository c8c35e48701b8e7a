#!/usr/bin/env python
"""Physics env-steps/s of the batched quadruped step on B200.

Workload (one "step" = one control step = 4 physics substeps of dt 0.005):
the procedural 12-DoF quadruped (free-joint trunk box, 4 legs x 3 hinges,
capsule links, sphere feet, position actuators kp 20 / kv 0.5), 16384 envs,
FP32, condim 3 pyramidal, self-collision on, Newton 16 iterations at
tolerance 1e-8, seeded uniform random position targets resampled every control
step.  Data are synthetic (seeded Philox), there is no dataset.

  value   whole-job env-steps/s with the per-step controls already resident in
          HBM (device-to-device copy into the sim, then the step kernel),
          CUDA events on the sim's stream, L2 flushed (256 MB write) before
          every timed step.
  e2e     the same metric through the public C ABI with host buffers:
          mjmlx_batched_step_n(ctrl host array, 4) + mjmlx_batched_get_state
          (qpos, qvel to host) every step, wall clock.
  roofline  the step kernel: algorithmic 488 B per env-substep (qpos, qvel,
          ctrl, warm-start qacc read; qpos, qvel, qacc written) over the
          kernel's CUDA-event time, against the measured HBM copy peak.
  cpu_baseline  the FP64 CPU oracle (a port of the step; MuJoCo C is not on
          the machine) on all host threads, bounded sample, rank 0 at N = 1.

--impl reference runs the reference-side CPU implementation that exists here
(the FP64 oracle port; the reference's own Vulkan/MuJoCo-C paths cannot be
built or run on this machine) on the same workload and prints its own line.
Multi-GPU (torchrun): independent replicas, one per GPU, no collective in the
physics; timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mujoco-mlx-cpp_b200"))

METRIC = "physics env-steps/s, 1 B200: plain vs learned warm-start, same solver tol"
UNIT = "env-steps/s"
SUBSTEPS = 4
BYTES_PER_ENV_SUBSTEP = 488  # qpos 76 + qvel 72 + ctrl 48 + warm qacc 72 read; qpos 76 + qvel 72 + qacc 72 written


def workload_config(B):
    return {
        "workload": f"quadruped12 (nq 19, nv 18, nu 12), {B} envs, 4 substeps x dt 0.005 per env-step, Newton max 16 it, tol 1e-8, "
                    "condim 3 pyramidal, self-collision on, random position targets resampled every env-step",
        "num_envs": B,
        "substeps_per_env_step": SUBSTEPS,
        "precision": "fp32 engine, fp64 oracle",
        "l2": "flushed before every timed step (256 MB write)",
        "data": "seeded synthetic initial states and controls (Philox)",
    }


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--envs", type=int, default=16384)
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    return ap.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    return world, rank, local


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic_per_env_launch():
    """Per-env DRAM bytes of one step-kernel launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "mjb_step_kernel_quadruped.md")
    try:
        with open(path) as f:
            for line in f:
                if line.strip().startswith("traffic_bytes_per_env_launch:"):
                    return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms in the background."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference(B, cpu_seconds, warmup=1):
    """FP64 oracle on all host threads: env-steps/s over a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mjb200
    import oracle

    nthread = os.cpu_count() or 1
    m = mjb200.load_model_from_string(mjb200.models.quadruped_xml())
    om = oracle.OracleModel(m.dump())
    Bs = min(B, 4096)
    ob = oracle.OracleBatch(om, Bs)
    q, v = mjb200.models.quadruped_initial_state_fast(Bs)
    ob.set_state(q, v)
    for w in range(warmup):
        ob.set_ctrl(mjb200.models.quadruped_controls_fast(Bs, w))
        ob.step(SUBSTEPS, nthread=nthread)
    n, t = 0, 0.0
    while t < cpu_seconds:
        ob.set_ctrl(mjb200.models.quadruped_controls_fast(Bs, warmup + n))
        t0 = time.perf_counter()
        ob.step(SUBSTEPS, nthread=nthread)
        t += time.perf_counter() - t0
        n += 1
    return {"value": Bs * n / t, "unit": UNIT, "cores": nthread, "kind": "port",
            "sample": f"{Bs} envs x {n} env-steps of the same workload, FP64 oracle (MuJoCo C absent), {nthread} host threads, {t:.1f} s"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    cb = cpu_reference(args.envs, args.cpu_seconds)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.envs), "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference CPU path = FP64 oracle port of the step (the reference's Vulkan GPU path and its MuJoCo C backend cannot run here)"}
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import mjb200
    from mjb200 import replicas

    torch.cuda.set_device(local)
    B = args.envs
    K, W = args.steps, args.warmup
    m = mjb200.load_model_from_string(mjb200.models.quadruped_xml())
    sim = mjb200.BatchedSim(m, B, record=0)
    seed_state, seed_ctrl = replicas.rank_seeds(rank)
    q0, v0 = mjb200.models.quadruped_initial_state_fast(B, seed=seed_state)
    nu = m.nu
    ctrl_all = np.stack([mjb200.models.quadruped_controls_fast(B, s, seed=seed_ctrl) for s in range(K + W)]).astype(np.float32)
    ctrl_dev = torch.from_numpy(ctrl_all).cuda()
    stride = B * nu
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    stream = torch.cuda.ExternalStream(sim.stream())

    def reset_state():
        sim.set_state(q0.astype(np.float32), v0.astype(np.float32))

    # ---- value: inputs resident in HBM
    reset_state()
    base = ctrl_dev.data_ptr()
    for w in range(W):
        sim.step_device_ctrl(base + 4 * w * stride, SUBSTEPS)
    sim.sync()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    niter_mean, niter_p99, ncon_mean = [], [], []
    with torch.cuda.stream(stream):
        for k in range(K):
            flush.zero_()
            a, b, c = ev[k]
            a.record(stream)
            sim.step_device_ctrl(base + 4 * (W + k) * stride, 0)
            b.record(stream)
            sim.step_device(SUBSTEPS)
            c.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(c) for a, b, c in ev]
    kern_ms = [b.elapsed_time(c) for a, b, c in ev]
    st = sim.stats()
    niter_mean = float(st["niter_sum"].mean() / SUBSTEPS)
    niter_p99 = float(np.percentile(st["niter_max"], 99))
    total_s = sum(step_ms) / 1e3
    total_s = replicas.reduce_over_ranks(total_s, "max", device="cuda")
    value = world * B * K / total_s

    # ---- e2e: public C ABI with host buffers
    reset_state()
    host_ctrl = [np.ascontiguousarray(ctrl_all[s]) for s in range(K + W)]
    for w in range(W):
        sim.step(host_ctrl[w], SUBSTEPS)
        sim.state()
    if world > 1:
        torch.distributed.barrier()
    e2e_s = 0.0
    for k in range(K):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.step(host_ctrl[W + k], SUBSTEPS)
        qp, qv = sim.state()
        e2e_s += time.perf_counter() - t0
    e2e_s = replicas.reduce_over_ranks(e2e_s, "max", device="cuda")
    e2e_value = world * B * K / e2e_s
    h2d = B * nu * 4
    d2h = B * (m.nq + m.nv) * 4

    # ---- roofline of the step kernel
    kern_s = statistics.mean(kern_ms) / 1e3
    alg_bytes = BYTES_PER_ENV_SUBSTEP * SUBSTEPS * B
    achieved = alg_bytes / kern_s / 1e9
    peak, peak_kind = peaks()
    tr = profile_traffic_per_env_launch()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": (tr * B) if tr is not None else None, "kernel": "mjb_step_kernel", "kernel_ms": statistics.mean(kern_ms),
                "algorithmic_bytes_per_launch": alg_bytes}

    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": 1e3 * total_s / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(B),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": roofline, "gpu_launches": K,
            "solver": {"warmstart": "previous-step (plain)", "newton_iter_mean": niter_mean, "newton_iter_p99": niter_p99,
                       "launch": sim.launch_shape()},
            "clocks": clocks}
    if world == 1:
        line["cpu_baseline"] = cpu_reference(B, args.cpu_seconds)
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
