#!/usr/bin/env python
"""Benchmark of the GRay2 geodesic hot path on B200.

Workload (default): torus_rt_1024 -- a=0.998 Kerr-Schild, 17 deg camera at
r=1000 M, 1024x1024 rays over +-20 M, RK4 with the reference step control
(64 dumps of -31.25 M with 1000 substeps: affine parameter 0 -> -2000 M),
radiative transfer at 4 frequencies through the analytic torus.  One bench
step = one full render (icond + every dump interval of every ray).

Metric: ray-steps/s = accepted RK4 steps summed over rays / time.
  value       mixed-precision persistent kernel, inputs resident in HBM,
              CUDA events on the launching stream, L2 flushed between steps
  fp64        the plain FP64 kernel (one launch per dump) on the same render
  e2e         the same metric through the C ABI with host buffers: render
              plus the device-to-host copy of the final state every step
  roofline    FP32 CUDA-core bound (the path has no dense contraction);
              peak = FMA-loop microbenchmark measured in this run
  cpu_baseline  the C oracle on the host cores, bounded ray sample

--impl reference times the reference's CPU implementation of the path:
the reference's OpenCL build cannot run here (no OpenCL platform, no lux
runtime, and its analytic Kerr-Schild kernel does not compile as shipped),
so its restatement in oracle/ (test/baseline infrastructure) is timed with
every host thread on a bounded sample of the same workload.

Multi-GPU (torchrun): every rank renders its own copy of the workload
(independent renders, weak scaling); the only collective is the max-over-
ranks of the timed region.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from gray_b200 import configs, flops  # noqa: E402

WORKLOADS = {"torus_rt_1024": configs.TORUS_RT_1024,
             "kerr_small_64": configs.KERR_SMALL_64,
             "numerical_128": configs.NUMERICAL_128,
             "survey_256": None,  # a batch of 256 renders (configs.survey)
             "serve_mix": None}   # Poisson request stream (configs.serve_requests)
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
METRIC = "ray-steps/s"

# DRAM bytes (read + write) of one full-size launch of the dominant kernel,
# from one-pass ncu captures (dram__bytes_read.sum + dram__bytes_write.sum).
TRAFFIC = {"torus_rt_1024": 145832704 + 116188928,
           "numerical_128": 500394240 + 17862656}
# Host-to-device bytes of one render through the C ABI: the render's table
# entry (sizeof(MixedRender) in gray_b200/csrc/mixed_table.h); the camera
# initial conditions are generated on the device.
H2D_BYTES_PER_RENDER = 392


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="torus_rt_1024", choices=sorted(WORKLOADS))
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--side", type=int, default=0, help="override the camera side (small runs)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--plan", default="measure", choices=["measure", "estimate", "rpt1", "rpt2"],
                    help="launch shape of the persistent kernel (measure = autotune)")
    ap.add_argument("--fp64-renders", type=int, default=16,
                    help="survey_256: renders run one at a time in FP64 for the comparison")
    ap.add_argument("--rates", default="0.5,1,2,3,4,6,8,12",
                    help="serve_mix: arrival rates (requests/s) swept in order")
    ap.add_argument("--requests", type=int, default=32, help="serve_mix: requests per rate")
    ap.add_argument("--partition", default="replicate", choices=["replicate", "split"],
                    help="survey_256 on N GPUs: every rank renders the survey (weak) or "
                         "the renders are split across ranks (strong)")
    ap.add_argument("--dumps-per-iter", type=int, default=16,
                    help="serve_mix: dump intervals each server iteration advances")
    return ap.parse_args()


# ------------------------------------------------------------------ CPU side

def cpu_rate(cfg, seconds, max_batches=10 ** 6):
    """Oracle ray-steps/s on every host thread over a strided ray sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    n_rays = cfg["n_width"] * cfg["n_height"]
    threads = os.cpu_count() or 1
    batch = max(threads * 2, 16)
    stride = 7919  # prime stride: rays from every part of the image
    done_steps, done_rays, t_used, k = 0, 0, 0.0, 0
    while (k == 0 or t_used < seconds) and k < max_batches:  # at least one batch
        rays = (np.arange(k * batch, (k + 1) * batch, dtype=np.int64) * stride) % n_rays
        t0 = time.perf_counter()
        _, _, steps = O.trace(cfg, rays, nthreads=threads)
        t_used += time.perf_counter() - t0
        done_steps += int(steps.sum())
        done_rays += batch
        k += 1
    return done_steps / t_used, threads, done_rays, t_used


def reference_arm(args, cfg, rank):
    if rank != 0:
        return
    per_step = max(args.cpu_seconds / max(args.steps, 1), 1.0)
    for _ in range(args.warmup):
        cpu_rate(cfg, 0.0, max_batches=1)
    rates, rays, secs = [], 0, 0.0
    threads = 1
    for _ in range(args.steps):
        r, threads, n, s = cpu_rate(cfg, per_step)
        rates.append(r)
        rays += n
        secs += s
    value = float(np.mean(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ray-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "rays_per_render": cfg["n_width"] * cfg["n_height"],
                   "sample": "strided rays", "precision": "fp64"},
        "cpu_baseline": {"value": value, "unit": "ray-steps/s", "cores": threads,
                         "kind": "port",
                         "sample": "%d rays of %s (stride 7919), every dump interval, %.1f s"
                                   % (rays, args.workload, secs)},
        "e2e": {"value": value, "unit": "ray-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.th.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        load = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ GPU side

def timed_renders(torch, render, k, flush):
    """k renders; per render events around icond+evolve and around evolve
    (the dominant kernel).  Returns (total_s, kernel_s)."""
    evs = []
    for _ in range(k):
        flush.zero_()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        render.icond()
        e1.record()
        render.evolve_all(wait=False)
        e2.record()
        evs.append((e0, e1, e2))
    torch.cuda.synchronize()
    tot = sum(a.elapsed_time(c) for a, b, c in evs) * 1e-3
    ker = sum(b.elapsed_time(c) for a, b, c in evs) * 1e-3
    return tot, ker


def max_over_ranks(torch, dist, x):
    """The slowest rank's time: the only collective of a multi-GPU run."""
    if dist is None:
        return x
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(torch, dist):
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()


def apply_plan(ctx, api, renders, how):
    """measure: autotune on these renders (gray_plan); estimate: the rule;
    rpt1/rpt2: force scalar or packed two-ray kernels."""
    if how in ("measure", "estimate"):
        b = ctx.batch(renders)
        try:
            p = ctx.plan(b, api.PLAN_MEASURE if how == "measure" else api.PLAN_ESTIMATE)
        finally:
            b.close()
        d = p.as_dict()
    else:
        ctx.set_plan(256 if how == "rpt1" else 128, 0, 1 if how == "rpt1" else 2)
        d = ctx.get_plan().as_dict()
    d["how"] = how
    return d


def ours_arm(args, cfg, rank, local_rank, world, dist):
    import torch
    from gray_b200 import api

    torch.cuda.set_device(local_rank)
    ctx = api.Context(local_rank)
    # One created stream for the library's launches and torch's events (the
    # legacy default stream has handle 0, which the C ABI reads as "use the
    # context's own stream").
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    nf = len(cfg.get("nu", ()))
    n_rays = cfg["n_width"] * cfg["n_height"]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    peak32 = ctx.measure_peak(api.PREC_MIXED)
    peak64 = ctx.measure_peak(api.PREC_FP64)

    # ---- mixed (headline); launch shape from the autotuner (gray_plan)
    rm = ctx.render(dict(cfg, precision=api.PREC_MIXED))
    plan = apply_plan(ctx, api, [rm], args.plan)
    for _ in range(args.warmup):
        rm.run()
    steps_per_render = rm.steps()
    barrier(torch, dist)
    clk = ClockSampler(local_rank)
    clk.start()
    tot, ker = timed_renders(torch, rm, args.steps, flush)
    clocks = clk.stop()
    barrier(torch, dist)
    tot = max_over_ranks(torch, dist, tot)
    ker = max_over_ranks(torch, dist, ker)
    value = world * steps_per_render * args.steps / tot
    mixed_state, mixed_info = rm.state(api.LAYOUT_SOA)

    flop_step = flops.mixed_per_step(nf)
    achieved = steps_per_render * flop_step / (ker / args.steps) / 1e12
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak32 / 1e12,
                "unit": "TFLOP/s", "frac": achieved * 1e12 / peak32,
                "traffic": None if args.side else TRAFFIC.get(args.workload),
                "peak_source": "FMA-loop microbenchmark in this run (best of scalar and f32x2 FFMA)",
                "flop_per_ray_step": flop_step,
                "kernel": "mixed_kernel<%d>" % nf}

    # ---- plain FP64 on the same render
    fp64 = None
    if not args.no_fp64:
        r64 = ctx.render(dict(cfg, precision=api.PREC_FP64))
        r64.run()  # warm-up
        s64 = r64.steps()
        barrier(torch, dist)
        t64, k64 = timed_renders(torch, r64, args.fp64_steps, flush)
        barrier(torch, dist)
        t64 = max_over_ranks(torch, dist, t64)
        k64 = max_over_ranks(torch, dist, k64)
        v64 = world * s64 * args.fp64_steps / t64
        st64, _ = r64.state(api.LAYOUT_SOA)
        img = {}
        for i in range(nf):
            ref = st64[8 + i]
            img["nu%g" % cfg["nu"][i]] = float(np.linalg.norm(mixed_state[8 + i] - ref) /
                                               np.linalg.norm(ref))
        pos = float(np.linalg.norm(mixed_state[1:4] - st64[1:4]) / np.linalg.norm(st64[1:4]))
        a64 = s64 * flops.fp64_per_step(nf) / (k64 / args.fp64_steps) / 1e12
        fp64 = {"value": v64, "unit": "ray-steps/s",
                "ms_per_step": 1e3 * t64 / args.fp64_steps,
                "ray_steps_per_render": s64,
                "mixed_over_fp64": value / v64,
                "image_rel_l2_err": img, "end_position_rel_l2_err": pos,
                "roofline": {"bound": "fp64", "achieved": a64, "peak": peak64 / 1e12,
                             "unit": "TFLOP/s", "frac": a64 * 1e12 / peak64,
                             "flop_per_ray_step": flops.fp64_per_step(nf)},
                "launches_per_render": 1 + int(cfg["n_dump"])}
        r64.close()

    # ---- end to end: render + device-to-host copy of the state, host buffers
    host = torch.empty((8 + 2 * nf) * n_rays, dtype=torch.float64, pin_memory=True).numpy()
    host = host.reshape(8 + 2 * nf, n_rays)
    hinfo = torch.empty(n_rays, dtype=torch.float64, pin_memory=True).numpy()
    rm.run()
    rm.state(api.LAYOUT_SOA, out=host, info_out=hinfo)
    barrier(torch, dist)
    e2e_t = 0.0
    for _ in range(args.e2e_steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rm.run(wait=False)
        rm.state(api.LAYOUT_SOA, out=host, info_out=hinfo)  # synchronous d2h
        e1.record()
        torch.cuda.synchronize()
        e2e_t += e0.elapsed_time(e1) * 1e-3
    barrier(torch, dist)
    e2e_t = max_over_ranks(torch, dist, e2e_t)
    e2e = {"value": world * steps_per_render * args.e2e_steps / e2e_t, "unit": "ray-steps/s",
           "h2d_bytes_per_step": H2D_BYTES_PER_RENDER,
           "d2h_bytes_per_step": int(host.nbytes + hinfo.nbytes)}
    rm.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, cores, rays, secs = cpu_rate(cfg, args.cpu_seconds)
        cpu = {"value": rate, "unit": "ray-steps/s", "cores": cores, "kind": "port",
               "sample": "%d rays of %s (stride 7919), every dump interval, %.1f s"
                         % (rays, args.workload, secs)}

    ctx.close()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "ray-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64-islands", "data": "synthetic",
        "config": {"workload": args.workload, "rays_per_render": n_rays,
                   "renders_per_gpu_per_step": 1, "n_freq": nf, "a_spin": cfg["a_spin"],
                   "i_obs": cfg["i_obs"], "affine_range": cfg["dt_dump"] * cfg["n_dump"],
                   "n_sub": cfg["n_sub"], "ray_steps_per_render": steps_per_render,
                   "precision": "mixed", "l2": "flushed (256 MiB write) between steps",
                   "parallelism": "independent renders per GPU" if world > 1 else "single GPU"},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": 2 * args.steps, "clocks": clocks, "fp64": fp64, "launch_plan": plan,
        "peaks_measured_tflops": {"fp32": peak32 / 1e12, "fp64": peak64 / 1e12},
    }
    print(json.dumps(line), flush=True)


def survey_arm(args, rank, local_rank, world, dist):
    """survey_256: 256 renders (32^2..512^2, random spin / inclination /
    distance, 4-frequency torus) as ONE batch: one graph-replayed persistent
    launch per step.  Compared with the FP64 kernel run one render at a time
    on the first --fp64-renders renders."""
    import torch
    from gray_b200 import api

    torch.cuda.set_device(local_rank)
    ctx = api.Context(local_rank)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    peak32 = ctx.measure_peak(api.PREC_MIXED)
    cfgs = configs.survey()
    scaling = "weak"
    if args.partition == "split" and world > 1:
        # strong scaling: the 256 renders are split across the ranks
        from gray_b200 import shard
        cfgs = shard.my_share(cfgs, [c["n_width"] * c["n_height"] for c in cfgs], rank, world)
        scaling = "strong"
    nf = len(cfgs[0]["nu"])
    rs = [ctx.render(dict(c, precision=api.PREC_MIXED)) for c in cfgs]
    n_rays = sum(r.n_rays for r in rs)
    plan = apply_plan(ctx, api, rs, args.plan)
    b = ctx.batch(rs)
    for _ in range(args.warmup):
        b.run()
    steps = b.steps()
    barrier(torch, dist)
    clk = ClockSampler(local_rank)
    clk.start()
    evs = []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.run(wait=False)
        e1.record()
        evs.append((e0, e1))
    torch.cuda.synchronize()
    clocks = clk.stop()
    tot = sum(a.elapsed_time(c) for a, c in evs) * 1e-3
    barrier(torch, dist)
    tot = max_over_ranks(torch, dist, tot)
    value = world * steps * args.steps / tot
    flop_step = flops.mixed_per_step(nf)
    achieved = steps * flop_step / (tot / args.steps) / 1e12
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak32 / 1e12,
                "unit": "TFLOP/s", "frac": achieved * 1e12 / peak32, "traffic": None,
                "peak_source": "FMA-loop microbenchmark in this run",
                "flop_per_ray_step": flop_step, "kernel": "mixed_kernel<%d> (batched)" % nf}

    # FP64, one render at a time, on a subset; image error of the batched mixed result
    fp64 = None
    if not args.no_fp64 and args.fp64_renders > 0:
        sub = list(range(min(args.fp64_renders, len(cfgs))))
        r0 = ctx.render(dict(cfgs[0], precision=api.PREC_FP64))
        r0.run()
        r0.close()
        t64, s64, errs = 0.0, 0, []
        for k in sub:
            r64 = ctx.render(dict(cfgs[k], precision=api.PREC_FP64))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            flush.zero_()
            e0.record()
            r64.run(wait=False)
            e1.record()
            torch.cuda.synchronize()
            t64 += e0.elapsed_time(e1) * 1e-3
            s64 += r64.steps()
            d64 = r64.state(api.LAYOUT_SOA)[0]
            dmx = rs[k].state(api.LAYOUT_SOA)[0]
            errs.append(max(float(np.linalg.norm(dmx[8 + i] - d64[8 + i]) / np.linalg.norm(d64[8 + i]))
                            for i in range(nf)))
            r64.close()
        v64 = s64 / t64
        fp64 = {"value": v64, "unit": "ray-steps/s", "renders": len(sub),
                "mode": "plain FP64 kernel, one render at a time",
                "mixed_batched_over_fp64_one_at_a_time": value / world / v64,
                "image_rel_l2_err_max": max(errs), "image_rel_l2_err_median": float(np.median(errs))}

    # end to end: batch + device-to-host copy of every render's state
    hosts = [torch.empty((r.n_data, r.n_rays), dtype=torch.float64, pin_memory=True).numpy()
             for r in rs]
    hinfo = [torch.empty(r.n_rays, dtype=torch.float64, pin_memory=True).numpy() for r in rs]
    barrier(torch, dist)
    e2e_t = 0.0
    for _ in range(args.e2e_steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.run(wait=False)
        for r, h, hi in zip(rs, hosts, hinfo):
            r.state(api.LAYOUT_SOA, out=h, info_out=hi)
        e1.record()
        torch.cuda.synchronize()
        e2e_t += e0.elapsed_time(e1) * 1e-3
    barrier(torch, dist)
    e2e_t = max_over_ranks(torch, dist, e2e_t)
    d2h = sum(h.nbytes for h in hosts) + sum(h.nbytes for h in hinfo)
    e2e = {"value": world * steps * args.e2e_steps / e2e_t, "unit": "ray-steps/s",
           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(d2h),
           "note": "render tables are uploaded once at batch creation; replays copy nothing in"}
    b.close()
    for r in rs:
        r.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, cores, rays, secs = cpu_rate(cfgs[len(cfgs) // 2], args.cpu_seconds)
        cpu = {"value": rate, "unit": "ray-steps/s", "cores": cores, "kind": "port",
               "sample": "%d rays of survey render %d (stride 7919), every dump interval, %.1f s"
                         % (rays, len(cfgs) // 2, secs)}
    ctx.close()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "ray-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": scaling, "vs_baseline": None,
        "dtype": "f32+f64-islands", "data": "synthetic",
        "config": {"workload": "survey_256", "renders": len(cfgs), "rays_per_step": n_rays,
                   "seed": configs.SURVEY_SEED, "n_freq": nf, "ray_steps_per_step": steps,
                   "precision": "mixed", "l2": "flushed (256 MiB write) between steps",
                   "graph": "one CUDA graph per step (256 icond + 1 persistent kernel)"},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": (len(cfgs) + 1) * args.steps, "clocks": clocks, "fp64": fp64,
        "launch_plan": plan,
    }
    print(json.dumps(line), flush=True)


GATHER_BYTES_PER_STEP = 4 * 2 * 8 * 40 * 4  # RHS x levels x corners x Gamma x float


def numerical_arm(args, cfg, rank, local_rank, world, dist):
    """numerical_128: boosted-KS 128^3 grid with two time levels (t = 0,
    10 M) over [-40, 40]^3, 512^2 camera at 200 M, mixed precision, physics
    mode (flat outside the box).  The kernel is gather-bound: roofline in
    algorithmic gather bytes (40 Gamma x 8 corners x 2 levels x 4 RHS per
    in-box step) against the measured HBM copy bandwidth."""
    import torch
    from gray_b200 import api

    torch.cuda.set_device(local_rank)
    ctx = api.Context(local_rank)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    G = configs.NUMERICAL_GRID
    grid = api.make_grid(G["n"], -G["box"], G["box"], G["t1"], G["t2"], physics=True)
    ctx.make_boosted_ks(grid, G["a"], G["v"], G["axis"], G["t1"], 0)
    ctx.make_boosted_ks(grid, G["a"], G["v"], G["axis"], G["t2"], 1)
    rm = ctx.render(dict(cfg, precision=api.PREC_MIXED))
    for _ in range(args.warmup):
        rm.run()
    steps, gsteps = rm.steps(), rm.gather_steps()
    barrier(torch, dist)
    clk = ClockSampler(local_rank)
    clk.start()
    tot, ker = timed_renders(torch, rm, args.steps, flush)
    clocks = clk.stop()
    barrier(torch, dist)
    tot = max_over_ranks(torch, dist, tot)
    ker = max_over_ranks(torch, dist, ker)
    value = world * steps * args.steps / tot
    mixed_state = rm.state(api.LAYOUT_SOA)[0]
    # end to end through the C ABI: each step renders from the camera on the
    # resident grid and reads the whole state back into pinned host memory
    n_rays = cfg["n_width"] * cfg["n_height"]
    host = torch.empty(8 * n_rays, dtype=torch.float64, pin_memory=True).numpy().reshape(8, n_rays)
    hinfo = torch.empty(n_rays, dtype=torch.float64, pin_memory=True).numpy()
    barrier(torch, dist)
    e2e_t = 0.0
    for _ in range(args.e2e_steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rm.run(wait=False)
        rm.state(api.LAYOUT_SOA, out=host, info_out=hinfo)  # synchronous d2h
        e1.record()
        torch.cuda.synchronize()
        e2e_t += e0.elapsed_time(e1) * 1e-3
    barrier(torch, dist)
    e2e_t = max_over_ranks(torch, dist, e2e_t)
    e2e = {"value": world * steps * args.e2e_steps / e2e_t, "unit": "ray-steps/s",
           "h2d_bytes_per_step": H2D_BYTES_PER_RENDER,
           "d2h_bytes_per_step": int(host.nbytes + hinfo.nbytes)}
    with open(MEASURED_PEAKS) as f:
        hbm = json.load(f)["hbm_gbs"]
    achieved = gsteps * GATHER_BYTES_PER_STEP / (ker / args.steps) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": None if args.side else TRAFFIC.get(args.workload),
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)",
                "bytes_per_gather_step": GATHER_BYTES_PER_STEP,
                "note": "algorithmic gather bytes; most hit L1/L2, so frac > 1 is cache reuse",
                "kernel": "dyst_mixed_kernel"}
    fp64 = None
    if not args.no_fp64:
        r64 = ctx.render(dict(cfg, precision=api.PREC_FP64))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r64.run(wait=False)
        e1.record()
        torch.cuda.synchronize()
        t64 = e0.elapsed_time(e1) * 1e-3
        s64 = r64.steps()
        ref = r64.state(api.LAYOUT_SOA)[0]
        r64.close()
        fin = np.all(np.isfinite(ref), axis=0) & np.all(np.isfinite(mixed_state), axis=0)
        # the image: rays that escaped to 100..1000 M; captured rays run on
        # inside the singular region (no horizon stop in dyst.cl:43-53) and
        # can leave it with absurd positions in either precision
        rend = np.sqrt(np.sum(ref[1:4] ** 2, axis=0))
        esc = fin & (rend > 100.0) & (rend < 1000.0)
        dpos = np.sqrt(np.sum((mixed_state[1:4, fin] - ref[1:4, fin]) ** 2, axis=0))
        fp64 = {"value": s64 / t64, "unit": "ray-steps/s", "ms_per_step": 1e3 * t64,
                "mixed_over_fp64": value / world / (s64 / t64),
                "end_position_abs_diff_median": float(np.median(dpos)),
                "end_position_abs_diff_p99": float(np.percentile(dpos, 99)),
                "end_position_abs_diff_max": float(dpos.max()),
                "ray_steps_fp64": s64,
                "end_position_rel_l2_err_escaping": float(
                    np.linalg.norm(mixed_state[1:4, esc] - ref[1:4, esc]) /
                    np.linalg.norm(ref[1:4, esc])),
                "escaping_fraction": float(esc.mean())}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        lv = [ctx.read_spacetime(grid, 0), ctx.read_spacetime(grid, 1)]
        og = O.Grid(lv, [G["t1"], -G["box"], -G["box"], -G["box"], G["t2"], G["box"], G["box"],
                         G["box"]], physics=True)
        threads = os.cpu_count() or 1
        batch, k, secs, done, nr = threads * 2, 0, 0.0, 0, 0
        while k == 0 or secs < args.cpu_seconds:
            rays = (np.arange(k * batch, (k + 1) * batch, dtype=np.int64) * 7919) % n_rays
            t0 = time.perf_counter()
            _, _, st = O.dyst_trace(cfg, og, rays, nthreads=threads)
            secs += time.perf_counter() - t0
            done += int(st.sum())
            nr += batch
            k += 1
        cpu = {"value": done / secs, "unit": "ray-steps/s", "cores": threads,
               "kind": "port", "sample": "%d rays of numerical_128 (stride 7919), %.1f s"
                                         % (nr, secs)}
    rm.close()
    ctx.close()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "ray-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64-islands", "data": "synthetic",
        "config": {"workload": "numerical_128", "grid": "128^3 x 2 levels FP32 boosted KS",
                   "rays_per_render": cfg["n_width"] * cfg["n_height"],
                   "ray_steps_per_render": steps, "gather_steps_per_render": gsteps,
                   "mode": "physics (flat outside the box, time factor clamped)",
                   "l2": "flushed (256 MiB write) between steps"},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": 2 * args.steps,
        "clocks": clocks, "fp64": fp64,
    }
    print(json.dumps(line), flush=True)


def serve_arm(args, rank, local_rank, world, dist):
    """serve_mix: seeded Poisson arrivals of analytic (70%) and numerical
    (30%) render requests into the continuous-batching server, with a
    device-resident 256^3 grid and a 120 GB admission budget.  The arrival
    rate is swept upward over the whole list; the sustained rate is the
    highest one whose p99 latency stays within 4x the p50 of the lowest
    rate (the unloaded latency), and `value` is the highest throughput of
    the sweep (the server's capacity on this mix)."""
    import time
    import torch
    from gray_b200 import api

    torch.cuda.set_device(local_rank)
    ctx = api.Context(local_rank)
    n = configs.SERVE_GRID_N
    grid = api.make_grid(n, -configs.SERVE_GRID_BOX, configs.SERVE_GRID_BOX, 0.0, 0.0, physics=True)
    ctx.make_boosted_ks(grid, 0.7, 0.3, 1, 0.0, 0)
    rates = [float(x) for x in args.rates.split(",")]
    # the same seeded request set at every rate, so the points compare
    reqs = configs.serve_requests(args.requests) * len(rates)
    rng = np.random.Generator(np.random.PCG64(configs.SERVE_SEED + 1))
    budget = int(120e9)
    ctx.serve_start(hbm_budget=budget, max_inflight=256, dumps_per_iter=args.dumps_per_iter)
    sweep, sustained, within, k0 = [], None, True, 0
    sample = {}  # class -> (cfg, served state) for the FP64 comparison
    try:
        # warm-up: one request of each kind
        first = {}
        for c in configs.serve_requests(32, seed=configs.SERVE_SEED + 2):
            first.setdefault(c.get("spacetime", 0), configs.scaled(c, 64))
        w = [ctx.submit(c) for c in first.values()]
        while any(ctx.poll(i).state < api.REQ_DONE for i in w):
            time.sleep(0.005)
        for i in w:
            ctx.release(i)
        for rate in rates:
            batch = reqs[k0:k0 + args.requests]
            k0 += args.requests
            gaps = rng.exponential(1.0 / rate, len(batch))
            s0, _ = ctx.serve_stats()
            steps0 = sum(s0.ray_steps)
            t_start = ctx.clock()
            due = t_start + np.cumsum(gaps)
            ids, pending = [], list(range(len(batch)))
            while pending:
                now = ctx.clock()
                if due[pending[0]] <= now:
                    j = pending.pop(0)
                    ids.append((ctx.submit(batch[j]), j))
                else:
                    time.sleep(min(0.002, due[pending[0]] - now))
            lat, kinds, t_end = [], [], t_start
            for rid, j in ids:
                while ctx.poll(rid).state < api.REQ_DONE:
                    time.sleep(0.002)
                s = ctx.poll(rid)
                lat.append(s.t_done - s.t_submit)
                t_end = max(t_end, s.t_done)
                kind = "numerical" if batch[j].get("spacetime") == 1 else "analytic"
                kinds.append(kind)
                if kind not in sample and batch[j]["n_width"] <= 256:
                    nd = 8 + 2 * len(batch[j]["nu"])
                    sample[kind] = (batch[j], ctx.result(rid, nd, s.n_rays)[0])
                else:
                    ctx.release(rid)
            s1, st = ctx.serve_stats()
            steps = sum(s1.ray_steps) - steps0
            lat = np.array(lat)
            p50, p99 = float(np.percentile(lat, 50)), float(np.percentile(lat, 99))
            row = {"rate_per_s": rate, "requests": len(batch), "p50_s": p50, "p99_s": p99,
                   "throughput": steps / (t_end - t_start), "wall_s": t_end - t_start,
                   "p50_by_class": {k: float(np.percentile(lat[np.array(kinds) == k], 50))
                                     for k in set(kinds)}}
            sweep.append(row)
            within &= p99 <= 4 * sweep[0]["p50_s"]
            if within:
                sustained = row
        stats, _ = ctx.serve_stats()
    finally:
        ctx.serve_stop()
    # mixed-vs-FP64 error per class on one sampled request each
    errs = {}
    for kind, (cfg, got) in sample.items():
        r = ctx.render(dict(cfg, precision=api.PREC_FP64))
        r.run()
        ref = r.state(api.LAYOUT_SOA)[0]
        r.close()
        if kind == "analytic":
            errs[kind] = {"image_rel_l2_err": max(float(np.linalg.norm(got[8 + i] - ref[8 + i]) /
                                                        np.linalg.norm(ref[8 + i])) for i in range(4))}
        else:
            # the numerical spacetime has no horizon stop (dyst.cl:43-53 gives
            # eps = 1), so captured rays run on inside the singular region where
            # FP32 and FP64 part ways; the image is the escaping rays (end
            # radius above 100 M in FP64)
            fin = np.all(np.isfinite(ref), axis=0) & np.all(np.isfinite(got), axis=0)
            rend = np.sqrt(np.sum(ref[1:4] ** 2, axis=0))
            esc = fin & (rend > 100.0) & (rend < 1000.0)
            errs[kind] = {"end_position_rel_l2_err_escaping": float(
                np.linalg.norm(got[1:4, esc] - ref[1:4, esc]) / np.linalg.norm(ref[1:4, esc])),
                "escaping_fraction": float(esc.mean())}
        errs[kind]["rays"] = int(ref.shape[1])
    ctx.close()
    if rank != 0:
        return
    best = sustained or sweep[0]
    peak = max(sweep, key=lambda r: r["throughput"])
    line = {
        "metric": METRIC, "value": peak["throughput"], "unit": "ray-steps/s", "n_gpus": world,
        "steps": len(sweep), "warmup": 1, "ms_per_step": 1e3 * peak["wall_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64-islands", "data": "synthetic",
        "config": {"workload": "serve_mix", "requests_per_rate": args.requests,
                   "grid": "%d^3 FP32 boosted KS (a=0.7, v=0.3 along x), %.2f GB" %
                           (n, n ** 3 * 56 * 4 / 1e9),
                   "hbm_budget_bytes": budget, "dumps_per_iter": args.dumps_per_iter,
                   "mix": "70% analytic torus 64..1024^2, 30% numerical 64..512^2"},
        "latency": {"p50_s": best["p50_s"], "p99_s": best["p99_s"],
                    "sustained_rate_per_s": best["rate_per_s"],
                    "rule": "highest rate with p99 <= 4 x the p50 of the lowest rate",
                    "unloaded_p50_s": sweep[0]["p50_s"],
                    "peak_throughput_rate_per_s": peak["rate_per_s"]},
        "sweep": sweep, "error_vs_fp64": errs,
        "serve_stats": {"iterations": stats.iterations, "busy_s": stats.busy_s,
                        "completed": stats.completed},
        "e2e": {"value": peak["throughput"], "unit": "ray-steps/s",
                "note": "request submit to result in host memory, host clock"},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "survey_256":
        # the reference arm samples the survey's median-index render
        cfg = configs.survey()[128]
    elif args.workload == "serve_mix":
        cfg = configs.serve_requests(8)[0]  # an analytic request of the stream
    else:
        cfg = dict(WORKLOADS[args.workload])
    if args.side:
        cfg = configs.scaled(cfg, args.side)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, cfg, rank)
        return
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as D
        torch.cuda.set_device(local_rank)
        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                             device_id=torch.device("cuda", local_rank))
        dist = D
    try:
        if args.workload == "survey_256":
            survey_arm(args, rank, local_rank, world, dist)
        elif args.workload == "serve_mix":
            serve_arm(args, rank, local_rank, world, dist)
        elif args.workload == "numerical_128":
            numerical_arm(args, cfg, rank, local_rank, world, dist)
        else:
            ours_arm(args, cfg, rank, local_rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
