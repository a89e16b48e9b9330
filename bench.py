#!/usr/bin/env python3
"""CG-SENSE reconstructions/s on B200: headline shape, 10 CG iterations, FP16x2 sparse MMA.

One step = one complete 10-iteration CG-SENSE reconstruction (adjoint right-hand side +
10 normal-operator applications, FP64 CG scalars) of the headline configuration:
256x256 image, 512x512 grid, 8 Gaussian-blob coils, golden-angle radial 256 spokes x 512
samples (131072 samples per coil), Kaiser-Bessel width 6.  Inputs are seeded synthetic
phantoms / coil maps / trajectories (the reference measures on OCMR, which is not
available); the measurement is the operator applied to the phantom plus 1e-3 rms noise.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config headline|cfg0|batch48|grad4]

--config batch48 reconstructs a seeded uneven batch of 48 cases per step through the batched
graph and reports the plain per-case drop-in (one solve after another) beside it.  The default
(headline) line also carries both comparisons, measured after the headline with 3 steps each
(--headline-only skips them).
--config grad4 times differentiable unrolled reconstructions (forward + hand-written backward,
gradients w.r.t. k-space data, coil maps and x0) of 4 cases per step.

Multi-GPU (torchrun, one process per GPU) runs independent replicas: every rank
reconstructs its own frames with no collective on the data path; value = all ranks'
reconstructions / max-over-ranks device time ("scaling": "weak").
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "CG-SENSE recons/s 256²x8coil x10CG at NRMSE<=0.2% vs FP64: batched/grad vs plain"
CONFIGS = {
    "headline": dict(n=256, g=512, c=8, spokes=256, readout=512, width=6, iters=10, density=False),
    "cfg0": dict(n=128, g=256, c=4, spokes=96, readout=256, width=6, iters=10, density=True),
    "batch48": dict(batch=True, cases=48, streams=4, width=6, iters=10),
    "grad4": dict(grad=True, cases=4, n=256, g=512, c=8, spokes=128, readout=512, width=6, iters=10, checkpoint=2,
                  density=False),
    "kooshball": dict(volume=True, n=128, g=256, c=8, spokes=16384, readout=256, width=4, iters=10),
    "vol64": dict(volume=True, n=64, g=128, c=8, spokes=2048, readout=128, width=4, iters=10),
}
VOLUME_METRIC = "CG-SENSE recons/s 128^3x8coil x10CG, 3D golden-means kooshball"
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def workload_text(cfg: dict) -> str:
    m = cfg["spokes"] * cfg["readout"]
    return (f"{cfg['n']}x{cfg['n']} image, {cfg['g']}x{cfg['g']} grid, {cfg['c']} coils, golden-angle radial "
            f"{cfg['spokes']}x{cfg['readout']} ({m} samples/coil), KB J={cfg['width']}, {cfg['iters']} CG iterations"
            + (", ramp density" if cfg["density"] else ""))


def synth_inputs(cfg: dict, seed: int):
    from trajsparsenufft_b200 import synth
    traj = synth.golden_radial(cfg["spokes"], cfg["readout"])
    x = synth.ellipse_phantom(cfg["n"], seed)
    s = synth.coil_maps(cfg["n"], cfg["c"], seed)
    w = synth.ramp_density(traj, cfg["readout"]) if cfg["density"] else None
    return traj, x, s, w


def nvml_handle(pynvml, index: int):
    """NVML handle of CUDA device `index` (matched by UUID: NVML numbers every GPU of the
    machine, CUDA only the visible ones)."""
    import torch
    uuid = str(torch.cuda.get_device_properties(index).uuid)
    try:
        return pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
    except Exception:
        return pynvml.nvmlDeviceGetHandleByIndex(index)


def gpu_local_cpus(index: int) -> set:
    """The CPUs NVML reports as local to CUDA device `index` (its NUMA node), within the ones
    this process may use; empty when NVML cannot say."""
    try:
        import pynvml
        pynvml.nvmlInit()
        h = nvml_handle(pynvml, index)
        words = pynvml.nvmlDeviceGetCpuAffinity(h, ((os.cpu_count() or 64) + 63) // 64)
        cpus = {64 * i + b for i, w in enumerate(words) for b in range(64) if (int(w) >> b) & 1}
        return cpus & os.sched_getaffinity(0)
    except Exception:
        return set()


class NumaLocal:
    """Allocates host buffers on the GPU's NUMA node: the calling thread runs on the GPU-local
    CPUs inside the block, so the pinned pages it touches first land on that node, and the
    copies to the device do not cross the inter-socket link. The thread's CPU set is restored
    afterwards (the CPU baseline keeps every core)."""

    def __init__(self, index: int):
        self.cpus = gpu_local_cpus(index)
        self.allowed = os.sched_getaffinity(0)

    def __enter__(self):
        if self.cpus and self.cpus != self.allowed:
            os.sched_setaffinity(0, self.cpus)
        return self

    def __exit__(self, *exc):
        if self.cpus and self.cpus != self.allowed:
            os.sched_setaffinity(0, self.allowed)
        return False

    def summary(self) -> dict:
        return {"gpu_local_cpus": len(self.cpus), "allowed_cpus": len(self.allowed),
                "pinned_on_gpu_node": bool(self.cpus)}


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while the timed region runs."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
        0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
        0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting",
    }

    def __init__(self, index: int):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = nvml_handle(pynvml, index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._nv = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for b, name in self.REASONS.items():
                    if bits & b and name != "gpu_idle":
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        if self._nv is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread is not None:
            self._thread.join()

    def summary(self) -> dict:
        med = statistics.median(self.samples) if self.samples else None
        return {"sm_mhz": med, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def max_over_ranks(ms: float, device) -> float:
    """Max of a per-rank device time over all ranks (the slowest replica sets the job time)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def median_run(run, device, repeats: int = 3):
    """Runs `run` (returning (device ms, extra)) `repeats` times; the max over ranks of each
    run's time, then the run with the median time: (ms, its extra, every run's ms).  One run
    of a host-copy loop can be slowed by traffic outside this process on the host's PCIe
    and memory, so the end-to-end figure is the median of several."""
    runs = []
    for _ in range(repeats):
        ms, extra = run()
        runs.append((max_over_ranks(ms, device), extra))
    ordered = sorted(runs, key=lambda r: r[0])
    ms, extra = ordered[len(ordered) // 2]
    return ms, extra, [r[0] for r in runs]


def job_rate(world: int, recons_per_step: int, steps: int, max_ms: float) -> float:
    """Whole-job reconstructions per second: every rank's reconstructions over the max time."""
    return world * recons_per_step * steps / (max_ms / 1e3)


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def committed_traffic(kernel: str):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get(kernel)
        except Exception:
            return None
    return None


def algorithmic_bytes(plan, cfg: dict) -> dict:
    """Compulsory HBM bytes of each stage per launch (reads + writes of an ideal design)."""
    info = plan.info
    n, g, c, m = cfg["n"], cfg["g"], cfg["c"], plan.samples
    panel_row = 8 * c            # FP16 hi + res, complex, C coils
    img = n * n * 8
    # inner CG iterations: the forward rows finish the previous update (r, p, ap, x in; x, r, p
    # out) and the inverse rows read r for the update's partials
    return {
        "fwd_rows": img * 7 + c * img + n * n * 4 + g * n * c * 8,          # r, p, ap, x rw, smaps, scaling, z1
        "fwd_cols": g * n * c * 8 + g * g * panel_row,                       # z1 read, panel write
        "interp_fwd": info["pack_bytes"][0] + g * g * panel_row + m * panel_row,   # pack, panel read, sample panel
        "interp_adj": info["pack_bytes"][1] + m * panel_row + info["active_rows"][1] * c * 8,  # pack, panel, grid
        "inv_cols": g * g * c * 8 + g * n * c * 8,
        "inv_rows": g * n * c * 8 + c * img + n * n * 4 + img * 3,          # w1, smaps, scaling, p, r, ap
        "cg_update": img * 6,                                                # the last iteration only
    }


def solve_bytes(alg: dict, iters: int, img: int, rhs: tuple) -> int:
    """Compulsory bytes of one solve: `iters` iterations whose forward rows (but the first)
    finish the previous update, one cg_update after the last, and the right-hand-side stages."""
    per_iter = sum(v for k, v in alg.items() if k != "cg_update")
    # the first forward rows reads r and writes p only; the last inverse rows reads no r
    return iters * per_iter - 5 * img - img + alg["cg_update"] + sum(alg[k] for k in rhs)


def run_ours(args, cfg) -> dict:
    import torch
    import torch.distributed as dist
    from trajsparsenufft_b200.operator import Plan

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    seed = 20260823 + rank
    traj, x_np, s_np, w_np = synth_inputs(cfg, seed)
    plan = Plan.from_trajectory(traj, im_size=cfg["n"], grid_size=cfg["g"], coils=cfg["c"], width=cfg["width"],
                                device=local, interp=args.interp)
    x_true = torch.from_numpy(x_np).to(dev)
    smaps = torch.from_numpy(s_np).to(dev)
    density = None if w_np is None else torch.from_numpy(w_np).to(dev)
    y_clean = plan.forward(x_true, smaps)
    g = torch.Generator(device=dev).manual_seed(seed)
    rms = y_clean.abs().pow(2).mean().sqrt()
    noise = torch.complex(torch.randn(y_clean.shape, device=dev, generator=g),
                          torch.randn(y_clean.shape, device=dev, generator=g))
    y = (y_clean + noise * (1e-3 * rms / math.sqrt(2.0))).contiguous()
    x_out = torch.empty_like(x_true)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    iters, lam = cfg["iters"], 1e-4

    def step():
        plan.cg_sense(y, smaps, density=density, lam=lam, iters=iters, out=x_out, sync=False)

    # correctness guard (host status once, outside the timed region)
    _, hist, status = plan.cg_sense(y, smaps, density=density, lam=lam, iters=iters, out=x_out, sync=True)
    if not (status["positive_curvature"] and status["finite"]):
        raise RuntimeError(f"CG status {status}")
    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        wall0 = time.perf_counter()
        for k in range(args.steps):
            flush.zero_()                      # L2 flushed between timed steps (not timed)
            starts[k].record()
            step()
            ends[k].record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        wall = time.perf_counter() - wall0
    dev_ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
    max_ms = max_over_ranks(dev_ms, dev)
    value = job_rate(world, 1, args.steps, max_ms)

    # end to end through the public call with host buffers: every step copies its y and maps
    # from pinned host memory and reads its image back.  The copy of step k+1 runs on a side
    # stream while step k solves (double-buffered device inputs); the L2 flush between steps
    # runs alone and its time is taken out of the total.
    numa = NumaLocal(local)
    with numa:
        y_h = y.cpu().pin_memory()
        s_h = smaps.cpu().pin_memory()
        x_hb = [torch.empty(x_out.shape, dtype=x_out.dtype).pin_memory() for _ in range(2)]
    y_d = [torch.empty_like(y) for _ in range(2)]
    s_d = [torch.empty_like(smaps) for _ in range(2)]
    e2e_steps = max(3, args.steps // 2)
    main = torch.cuda.current_stream()
    side = torch.cuda.Stream(device=dev)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    # the image read-back is double-buffered too: step k's image leaves on a second side stream
    # while step k+1 solves (after that step's flush, which is taken out of the total)
    x_d = [x_out, torch.empty_like(x_out)]
    down = torch.cuda.Stream(device=dev)

    def e2e_run(nsteps):
        copy0 = [ev() for _ in range(nsteps)]
        copied = [ev() for _ in range(nsteps)]
        f0 = [ev() for _ in range(nsteps)]
        f1 = [ev() for _ in range(nsteps)]
        read = [ev() for _ in range(nsteps)]
        start, end = ev(), ev()
        start.record(main)
        side.wait_stream(main)
        down.wait_stream(main)
        with torch.cuda.stream(side):
            copy0[0].record(side)
            y_d[0].copy_(y_h, non_blocking=True)
            s_d[0].copy_(s_h, non_blocking=True)
            copied[0].record(side)
        for k in range(nsteps):
            b = k & 1
            main.wait_event(copied[k])     # inputs of step k are on the device; the next copy is done
            if k >= 2:
                main.wait_event(read[k - 2])  # x_d[b] has been read back
            f0[k].record(main)
            flush.zero_()
            f1[k].record(main)
            if k >= 1:                     # the previous image streams out while this step solves
                down.wait_event(f1[k])
                with torch.cuda.stream(down):
                    x_hb[b ^ 1].copy_(x_d[b ^ 1], non_blocking=True)
                    read[k - 1].record(down)
            if k + 1 < nsteps:             # next inputs stream in while this step solves
                side.wait_event(f1[k])
                with torch.cuda.stream(side):
                    copy0[k + 1].record(side)
                    y_d[b ^ 1].copy_(y_h, non_blocking=True)
                    s_d[b ^ 1].copy_(s_h, non_blocking=True)
                    copied[k + 1].record(side)
            plan.cg_sense(y_d[b], s_d[b], density=density, lam=lam, iters=iters, out=x_d[b], sync=False)
        last = (nsteps - 1) & 1
        down.wait_stream(main)
        with torch.cuda.stream(down):
            x_hb[last].copy_(x_d[last], non_blocking=True)
            read[nsteps - 1].record(down)
        main.wait_stream(down)
        end.record(main)
        torch.cuda.synchronize()
        flush_ms = sum(a.elapsed_time(b_) for a, b_ in zip(f0, f1))
        h2d_ms = statistics.median(a.elapsed_time(b_) for a, b_ in zip(copy0, copied))
        return start.elapsed_time(end) - flush_ms, h2d_ms

    e2e_run(2)
    e2e_ms, h2d_ms, e2e_repeats = median_run(lambda: e2e_run(e2e_steps), dev)
    e2e_value = job_rate(world, 1, e2e_steps, e2e_ms)

    # dominant kernel: per-stage CUDA-event timing on this stream
    stages = plan.profile_stages(y, smaps, reps=20)
    alg = algorithmic_bytes(plan, cfg)
    dominant = max(stages, key=stages.get)
    peak, peak_kind = measured_peaks()
    achieved = alg[dominant] / (stages[dominant] * 1e-3) / 1e9
    per_iter_ms = sum(v for k, v in stages.items() if k != "cg_update")
    recon_bytes = solve_bytes(alg, iters, cfg["n"] ** 2 * 8, ("interp_adj", "inv_cols", "inv_rows"))
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "recons/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f16x2->f32 (f64 CG scalars)", "data": "synthetic",
        "config": {"workload": workload_text(cfg), "samples_per_coil": plan.samples, "recons_per_step": 1,
                   "l2": "flushed between timed steps (256 MB write)", "parallelism": f"replicas x{world}",
                   "planner": "optimized/morton split24", "pack": "real KB coefficients, centred image",
                   "interp_kernel": plan.interp,
                   "tiles": plan.info["tiles"], "groups": plan.info["groups"]},
        "e2e": {"value": round(e2e_value, 3), "unit": "recons/s",
                "h2d_bytes_per_step": int(y.numel() * 8 + smaps.numel() * 8),
                "d2h_bytes_per_step": int(x_out.numel() * 8),
                "overlap": "the input copy of step k+1 and the image read-back of step k-1 overlap the solve of step k",
                "h2d_ms_per_step": round(h2d_ms, 4),
                "repeats": [round(job_rate(world, 1, e2e_steps, m), 3) for m in e2e_repeats],
                "statistic": f"median of {len(e2e_repeats)} runs of {e2e_steps} steps",
                "host_buffers": numa.summary()},
        "gpu_launches": args.steps * (5 + 6 * iters + 2),
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1), "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": committed_traffic(dominant),
                     "algorithmic_bytes_per_launch": alg[dominant], "launch_ms": round(stages[dominant], 5)},
        "step_roofline": {"algorithmic_bytes_per_recon": int(recon_bytes),
                          "achieved_GBs": round(recon_bytes * value / world / 1e9, 1),
                          "frac": round(recon_bytes * value / world / 1e9 / peak, 4)},
        "stage_ms": {k: round(v, 5) for k, v in stages.items()},
        "per_iteration_stage_sum_ms": round(per_iter_ms, 4),
        "wall_s": round(wall, 3),
        "clocks": clocks.summary(),
        "residual_ratio": hist[-1] / hist[0],
    }
    out["nonuniform_samples_per_s"] = round(value * cfg["c"] * plan.samples * iters * 2, 1)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"], out["accuracy"] = cpu_checks(cfg, traj, x_np, s_np, y.cpu().numpy(),
                                                          y_clean.cpu().numpy(), x_out.cpu().numpy(), density)
    if rank == 0 and world == 1 and not args.headline_only:
        out.update(side_configs(args))
    return out if rank == 0 else None


def side_configs(args) -> dict:
    """The metric's "batched/grad vs plain" half, measured after the headline in the same run:
    the 48-case uneven batch (batched graph against the plain per-case drop-in) and the
    differentiable 4-case unrolled recon (gradients against the forward-only and the plain
    graph solver), each with 3 warm-up and 3 timed steps of its own configuration."""
    import copy
    sub = copy.copy(args)
    sub.steps, sub.warmup = 3, 3
    b = run_batch(sub, dict(CONFIGS["batch48"]))
    g = run_grad(sub, dict(CONFIGS["grad4"]))
    return {
        "batched_vs_plain": {
            "config": b["config"]["workload"], "batched_recons_per_s": b["value"],
            "plain_per_case_recons_per_s": b["plain_per_case"]["value"], "ratio": b["batch_speedup"],
            "nonuniform_samples_per_s": b["nonuniform_samples_per_s"], "plan_seconds": b["config"]["plan_seconds"],
            "steps": sub.steps, "warmup": sub.warmup},
        "grad_vs_plain": {
            "config": g["config"]["workload"], "recons_per_s_with_gradients": g["value"],
            "forward_only_recons_per_s": g["forward_only"]["value"],
            "plain_graph_solver_recons_per_s": g["plain_graph_solver"]["value"],
            "backward_over_forward": g["backward_over_forward"],
            "ratio_with_gradients_over_plain": round(g["value"] / g["plain_graph_solver"]["value"], 4),
            "steps": sub.steps, "warmup": sub.warmup},
    }


def cpu_checks(cfg, traj, x_np, s_np, y_np, y_clean_gpu, x_gpu, density) -> tuple[dict, dict]:
    """On the host, outside every timed region: (1) the CPU baseline -- full 10-iteration FP32
    CG-SENSE solves of the same workload by the CPU path restated from the reference's
    reference_sparse_solver (fp32/fp32 CSR), timed on all host cores; (2) the accuracy of the
    GPU reconstruction just timed: magnitude NRMSE against the FP64 KB CG of the same k-space
    (and against the phantom), and the GPU forward operator against the FP64 direct NUDFT on
    every 64th sample."""
    from oracle import nudft
    from oracle import operator as oop
    from oracle.cpu_ref import CpuSenseFp32
    threads = os.cpu_count() or 1
    w_np = None if density is None else density.cpu().numpy().astype(np.float64)
    op = CpuSenseFp32(traj, cfg["n"], cfg["g"], cfg["width"], s_np, threads=threads)
    yw = y_np if w_np is None else (y_np * w_np[None]).astype(np.complex64)
    times = []
    for _ in range(2):
        t0 = time.perf_counter()
        op.cg_sense(yw, cfg["iters"], 1e-4)
        times.append(time.perf_counter() - t0)
    t_recon = min(times)
    base = {"value": round(1.0 / t_recon, 5), "unit": "recons/s", "cores": threads, "kind": "port",
            "sample": f"2 full {cfg['iters']}-iteration FP32 CG-SENSE solves of the same workload (the "
                      "reference_sparse_solver fp32/fp32 CSR path restated; its operator and CG pinned to the "
                      "reference's own output in tests/golden/solver_small.npz), best of 2",
            "seconds_per_recon": round(t_recon, 3)}
    f64 = oop.KbSenseOperator(traj, cfg["n"], cfg["g"], cfg["width"], workers=threads)
    adj = (lambda v: f64.adjoint(v, s_np)) if w_np is None else (lambda v: f64.adjoint(v * w_np[None], s_np))
    x_ref, _, _ = oop.cg_sense(lambda v: f64.forward(v, s_np), adj, y_np.astype(np.complex128), cfg["iters"], 1e-4)
    sub = np.arange(0, len(traj), 64)
    exact = nudft.Nudft(traj[sub], cfg["n"]).forward(x_np, s_np)
    fwd_err = float(np.linalg.norm(y_clean_gpu[:, sub] - exact) / np.linalg.norm(exact))
    acc = {"recon_magnitude_nrmse_vs_fp64_cg": round(oop.magnitude_nrmse(x_gpu, x_ref), 7),
           "recon_rel_l2_vs_fp64_cg": round(oop.nrmse(x_gpu, x_ref), 7),
           "fp64_cg": f"FP64 Kaiser-Bessel (J={cfg['width']}) CG-SENSE, {cfg['iters']} iterations, same k-space",
           "recon_magnitude_nrmse_vs_phantom": round(oop.magnitude_nrmse(x_gpu, x_np), 5),
           "forward_rel_l2_vs_fp64_nudft": round(fwd_err, 7), "nudft_subsample": int(len(sub)),
           "gate": "recon magnitude NRMSE <= 2e-3 (0.2%)"}
    return base, acc


def run_batch(args, cfg) -> dict | None:
    """Uneven 48-case batch: the batched graph (tsn_batch_cg_sense) against the plain per-case
    drop-in (one tsn_cg_sense graph per case, back to back on one stream), same inputs."""
    import torch
    from concurrent.futures import ThreadPoolExecutor
    from trajsparsenufft_b200 import synth
    from trajsparsenufft_b200.operator import Batch, Plan

    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    specs = synth.uneven_batch(cfg["cases"], 20260823 + 1000 * rank)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=4) as ex:  # ctypes releases the GIL; the planner threads inside
        plans = list(ex.map(lambda sp: Plan.from_trajectory(sp["trajectory"], im_size=sp["n"], grid_size=sp["g"],
                                                            coils=sp["c"], width=cfg["width"], device=local), specs))
    plan_s = time.perf_counter() - t0
    ys, maps = [], []
    for sp, pl in zip(specs, plans):
        x = torch.from_numpy(synth.ellipse_phantom(sp["n"], sp["seed"])).to(dev)
        s = torch.from_numpy(synth.coil_maps(sp["n"], sp["c"], sp["seed"])).to(dev)
        yc = pl.forward(x, s)
        g = torch.Generator(device=dev).manual_seed(sp["seed"])
        rms = yc.abs().pow(2).mean().sqrt()
        noise = torch.complex(torch.randn(yc.shape, device=dev, generator=g),
                              torch.randn(yc.shape, device=dev, generator=g))
        ys.append((yc + noise * (1e-3 * rms / math.sqrt(2.0))).contiguous())
        maps.append(s)
    outs = [torch.empty((sp["n"], sp["n"]), dtype=torch.complex64, device=dev) for sp in specs]
    iters, lam = cfg["iters"], 1e-4
    batch = Batch(plans, streams=cfg["streams"])
    _, statuses = batch.cg_sense(ys, maps, lam=lam, iters=iters, outs=outs, sync=True)
    bad = [i for i, st in enumerate(statuses) if "failure" in st]
    if bad:
        raise RuntimeError(f"CG status failure in cases {bad}")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def plain_step():
        for pl, y, s, o in zip(plans, ys, maps, outs):
            pl.cg_sense(y, s, lam=lam, iters=iters, out=o, sync=False)

    def batch_step():
        batch.cg_sense(ys, maps, lam=lam, iters=iters, outs=outs, sync=False)

    def timed(step):
        for _ in range(args.warmup):
            flush.zero_()
            step()
        torch.cuda.synchronize()
        st = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        en = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            st[k].record()
            step()
            en[k].record()
        torch.cuda.synchronize()
        return max_over_ranks(sum(a.elapsed_time(b) for a, b in zip(st, en)), dev)

    plain_ms = timed(plain_step)
    with ClockSampler(local) as clocks:
        batch_ms = timed(batch_step)
    n_cases = len(specs)
    value = job_rate(world, n_cases, args.steps, batch_ms)
    plain_value = job_rate(world, n_cases, args.steps, plain_ms)

    # end to end: every step copies all cases' y and maps from pinned host memory (side stream,
    # overlapping the previous step's solve) and reads every image back
    with NumaLocal(local):
        y_h = [y.cpu().pin_memory() for y in ys]
        s_h = [s.cpu().pin_memory() for s in maps]
        x_h = [torch.empty(o.shape, dtype=o.dtype).pin_memory() for o in outs]
    y_d = [[torch.empty_like(y) for y in ys] for _ in range(2)]
    s_d = [[torch.empty_like(s) for s in maps] for _ in range(2)]
    main = torch.cuda.current_stream()
    side = torch.cuda.Stream(device=dev)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def copy_in(b):
        for a, h in zip(y_d[b], y_h):
            a.copy_(h, non_blocking=True)
        for a, h in zip(s_d[b], s_h):
            a.copy_(h, non_blocking=True)

    def e2e_run(nsteps):
        copied = [ev() for _ in range(nsteps + 1)]
        f0 = [ev() for _ in range(nsteps)]
        f1 = [ev() for _ in range(nsteps)]
        start, end = ev(), ev()
        start.record(main)
        side.wait_stream(main)
        with torch.cuda.stream(side):
            copy_in(0)
            copied[0].record(side)
        for k in range(nsteps):
            b = k & 1
            main.wait_event(copied[k])
            f0[k].record(main)
            flush.zero_()
            f1[k].record(main)
            if k + 1 < nsteps:
                side.wait_event(f1[k])
                with torch.cuda.stream(side):
                    copy_in(b ^ 1)
                    copied[k + 1].record(side)
            batch.cg_sense(y_d[b], s_d[b], lam=lam, iters=iters, outs=outs, sync=False)
            for h, o in zip(x_h, outs):
                h.copy_(o, non_blocking=True)
        end.record(main)
        torch.cuda.synchronize()
        return start.elapsed_time(end) - sum(a.elapsed_time(b_) for a, b_ in zip(f0, f1)), None

    e2e_steps = max(3, args.steps // 2)
    e2e_run(2)
    e2e_ms, _, e2e_repeats = median_run(lambda: e2e_run(e2e_steps), dev)
    e2e_value = job_rate(world, n_cases, e2e_steps, e2e_ms)
    if world > 1:
        torch.distributed.destroy_process_group()
    samples = sum(len(sp["trajectory"]) * sp["c"] for sp in specs)
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "recons/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(batch_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f16x2->f32 (f64 CG scalars)", "data": "synthetic",
        "config": {"workload": f"uneven batch of {n_cases} cases per step (synth.uneven_batch): N in "
                               "{128,192,256,320} (grid 2N), coils in {4,8,12,16}, half golden-angle radial "
                               "(64-384 spokes x 2N), half variable-density spirals (8-32 x 2048-4096), KB J=6, "
                               f"{iters} CG iterations",
                   "cases": n_cases, "streams": cfg["streams"], "recons_per_step": n_cases,
                   "l2": "flushed between timed steps (256 MB write)", "parallelism": f"replicas x{world}",
                   "plan_seconds": round(plan_s, 1)},
        "plain_per_case": {"value": round(plain_value, 3), "unit": "recons/s",
                           "ms_per_step": round(plain_ms / args.steps, 4)},
        "batch_speedup": round(value / plain_value, 3),
        "nonuniform_samples_per_s": round(value / n_cases * samples * iters * 2, 1),
        "e2e": {"value": round(e2e_value, 3), "unit": "recons/s",
                "h2d_bytes_per_step": int(sum(y.numel() * 8 for y in ys) + sum(s.numel() * 8 for s in maps)),
                "d2h_bytes_per_step": int(sum(o.numel() * 8 for o in outs)),
                "overlap": "copies of step k+1 overlap the solve of step k",
                "repeats": [round(job_rate(world, n_cases, e2e_steps, m), 3) for m in e2e_repeats],
                "statistic": f"median of {len(e2e_repeats)} runs of {e2e_steps} steps"},
        "gpu_launches": args.steps * n_cases * (5 + 6 * iters + 2),
        "clocks": clocks.summary(),
    }
    return out if rank == 0 else None


def run_grad(args, cfg) -> dict | None:
    """Differentiable unrolled reconstructions: loss = sum_i |x_i - x_true_i|^2 after 10 CG-SENSE
    iterations of each case, gradients w.r.t. k-space data, coil maps and x0 (autograd.py)."""
    import torch
    from trajsparsenufft_b200 import autograd as tad
    from trajsparsenufft_b200 import synth
    from trajsparsenufft_b200.operator import Plan

    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    n, g, c = cfg["n"], cfg["g"], cfg["c"]
    traj = synth.golden_radial(cfg["spokes"], cfg["readout"])
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=cfg["width"], device=local)
    ops = tad.PlanOps(plan)
    iters, lam, every = cfg["iters"], 1e-4, cfg["checkpoint"]
    xts, maps, ys = [], [], []
    for i in range(cfg["cases"]):
        seed = 20260823 + 100 * rank + i
        xt = torch.from_numpy(synth.ellipse_phantom(n, seed)).to(dev)
        s = torch.from_numpy(synth.coil_maps(n, c, seed)).to(dev)
        yc = plan.forward(xt, s)
        gen = torch.Generator(device=dev).manual_seed(seed)
        rms = yc.abs().pow(2).mean().sqrt()
        noise = torch.complex(torch.randn(yc.shape, device=dev, generator=gen),
                              torch.randn(yc.shape, device=dev, generator=gen))
        ys.append((yc + noise * (1e-3 * rms / math.sqrt(2.0))).contiguous())
        xts.append(xt)
        maps.append(s)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    outs = [torch.empty((n, n), dtype=torch.complex64, device=dev) for _ in ys]

    def grad_step(y_in=None, s_in=None):
        y_in = ys if y_in is None else y_in
        s_in = maps if s_in is None else s_in
        leaves = []
        loss = 0.0
        for y, s, xt in zip(y_in, s_in, xts):
            yl = y.detach().requires_grad_(True)
            sl = s.detach().requires_grad_(True)
            x0 = torch.zeros((n, n), dtype=torch.complex64, device=dev, requires_grad=True)
            xk = tad.cg_sense(yl, sl, ops, x0=x0, lam=lam, iters=iters, checkpoint=every)
            loss = loss + (xk - xt).abs().pow(2).sum()
            leaves.append((yl, sl, x0))
        loss.backward()
        return loss, leaves

    def fwd_step():
        with torch.no_grad():
            for y, s in zip(ys, maps):
                tad.cg_sense(y, s, ops, lam=lam, iters=iters, checkpoint=every)

    def plain_step():
        for y, s, o in zip(ys, maps, outs):
            plan.cg_sense(y, s, lam=lam, iters=iters, out=o, sync=False)

    def timed(step):
        for _ in range(args.warmup):
            flush.zero_()
            step()
        torch.cuda.synchronize()
        st = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        en = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            st[k].record()
            step()
            en[k].record()
        torch.cuda.synchronize()
        return max_over_ranks(sum(a.elapsed_time(b) for a, b in zip(st, en)), dev)

    eager_grad_ms = timed(grad_step)
    eager_fwd_ms = timed(fwd_step)
    plain_ms = timed(plain_step)

    # The whole gradient step (all cases' forward solves, the loss and the backward) as one
    # CUDA graph: static input tensors, leaves made once, grads allocated at capture and
    # overwritten by every replay.
    y_st = [y.clone() for y in ys]
    s_st = [s.clone() for s in maps]
    yl = [y.detach().requires_grad_(True) for y in y_st]
    sl = [s.detach().requires_grad_(True) for s in s_st]
    x0l = [torch.zeros((n, n), dtype=torch.complex64, device=dev, requires_grad=True) for _ in ys]
    leaves = yl + sl + x0l

    def graph_body():
        loss = 0.0
        for y, s, x0, xt in zip(yl, sl, x0l, xts):
            xk = tad.cg_sense(y, s, ops, x0=x0, x0_zero=True, lam=lam, iters=iters, checkpoint=every)
            loss = loss + (xk - xt).abs().pow(2).sum()
        loss.backward()
        return loss

    def fwd_body():
        with torch.no_grad():
            return [tad.cg_sense(y, s, ops, lam=lam, iters=iters, checkpoint=every) for y, s in zip(y_st, s_st)]

    def capture(body, clear_grads):
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(3):
                if clear_grads:
                    for leaf in leaves:
                        leaf.grad = None
                body()
        torch.cuda.current_stream().wait_stream(side)
        if clear_grads:
            for leaf in leaves:
                leaf.grad = None
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, capture_error_mode="relaxed"):
            result = body()
        return graph, result

    g_grad, g_loss = capture(graph_body, True)
    g_fwd, _ = capture(fwd_body, False)
    # the graph replays the eager step's kernels: its gradients match an eager step's
    g_grad.replay()
    _, leaves_e = grad_step()
    torch.cuda.synchronize()
    eager_leaves = [trip[k] for k in range(3) for trip in leaves_e]  # all y, all maps, all x0: as `leaves`
    graph_vs_eager = max(
        float(torch.linalg.vector_norm(a.grad - b.grad) / torch.linalg.vector_norm(b.grad).clamp_min(1e-30))
        for a, b in zip(leaves, eager_leaves))
    with ClockSampler(local) as clocks:
        grad_ms = timed(g_grad.replay)
    fwd_ms = timed(g_fwd.replay)

    # end to end: inputs from pinned host memory into the graph's static inputs, then the loss
    # and every gradient back to the host
    with NumaLocal(local):
        y_h = [y.cpu().pin_memory() for y in ys]
        s_h = [s.cpu().pin_memory() for s in maps]
        grads_h = [torch.empty(leaf.shape, dtype=leaf.dtype).pin_memory() for leaf in leaves]
        loss_h = torch.empty((), dtype=g_loss.dtype).pin_memory()

    def e2e_step():
        for dst, h in zip(y_st + s_st, y_h + s_h):
            dst.copy_(h, non_blocking=True)
        g_grad.replay()
        loss_h.copy_(g_loss.detach(), non_blocking=True)
        for h, leaf in zip(grads_h, leaves):
            h.copy_(leaf.grad, non_blocking=True)

    def e2e_run(nsteps):
        es = [torch.cuda.Event(enable_timing=True) for _ in range(nsteps)]
        ee = [torch.cuda.Event(enable_timing=True) for _ in range(nsteps)]
        for k in range(nsteps):
            flush.zero_()
            es[k].record()
            e2e_step()
            ee[k].record()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in zip(es, ee)), None

    e2e_steps = max(3, args.steps // 2)
    e2e_run(2)
    e2e_ms, _, e2e_repeats = median_run(lambda: e2e_run(e2e_steps), dev)
    if world > 1:
        torch.distributed.destroy_process_group()
    cases = cfg["cases"]
    value = job_rate(world, cases, args.steps, grad_ms)
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "recons/s (with gradients)", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(grad_ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16x2->f32 (f64 CG scalars)",
        "data": "synthetic",
        "config": {"workload": f"{cases} cases per step: {n}x{n} image, {g}x{g} grid, {c} coils, golden-angle "
                               f"radial {cfg['spokes']}x{cfg['readout']}, KB J={cfg['width']}, {iters} unrolled "
                               f"CG-SENSE iterations (checkpoint every {every}); loss |x - x_true|^2, gradients "
                               "w.r.t. k-space data, coil maps and x0",
                   "recons_per_step": cases, "l2": "flushed between timed steps (256 MB write)",
                   "parallelism": f"replicas x{world}",
                   "step": "one CUDA graph per step: forward solves, loss and backward of all cases"},
        "forward_only": {"value": round(job_rate(world, cases, args.steps, fwd_ms), 3), "unit": "recons/s",
                         "ms_per_step": round(fwd_ms / args.steps, 4)},
        "backward_over_forward": round((grad_ms - fwd_ms) / fwd_ms, 3),
        "graph_grads_rel_diff_vs_eager": graph_vs_eager,
        "eager": {"value": round(job_rate(world, cases, args.steps, eager_grad_ms), 3),
                  "ms_per_step": round(eager_grad_ms / args.steps, 4),
                  "forward_only_ms_per_step": round(eager_fwd_ms / args.steps, 4),
                  "backward_over_forward": round((eager_grad_ms - eager_fwd_ms) / eager_fwd_ms, 3)},
        "plain_graph_solver": {"value": round(job_rate(world, cases, args.steps, plain_ms), 3),
                               "unit": "recons/s", "ms_per_step": round(plain_ms / args.steps, 4)},
        "e2e": {"value": round(job_rate(world, cases, e2e_steps, e2e_ms), 3),
                "unit": "recons/s (with gradients)",
                "h2d_bytes_per_step": int(sum(y.numel() * 8 for y in ys) + sum(s.numel() * 8 for s in maps)),
                "d2h_bytes_per_step": int(8 + sum(leaf.numel() * 8 for leaf in leaves)),
                "repeats": [round(job_rate(world, cases, e2e_steps, v), 3) for v in e2e_repeats],
                "statistic": f"median of {len(e2e_repeats)} runs of {e2e_steps} steps"},
        "gpu_launches": None,
        "clocks": clocks.summary(),
    }
    return out if rank == 0 else None


def run_reference(args, cfg) -> dict | None:
    """Reference arm: the reference's CPU FP32 CG-SENSE path (restated port) on host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    if cfg.get("volume"):
        return {"impl": "reference", "unavailable": "the reference path is 2D only (no volume NUFFT to run)"}
    from oracle.cpu_ref import CpuSenseFp32
    threads = os.cpu_count() or 1
    if cfg.get("batch"):  # a bounded sample: the first cases of the batch, one per step in turn
        from trajsparsenufft_b200 import synth
        specs = synth.uneven_batch(cfg["cases"], 20260823)[:4]
        cases = [(sp["trajectory"], synth.ellipse_phantom(sp["n"], sp["seed"]),
                  synth.coil_maps(sp["n"], sp["c"], sp["seed"]), sp["n"], sp["g"]) for sp in specs]
        workload = f"cases 0-3 of the {cfg['cases']}-case uneven batch (synth.uneven_batch)"
    else:
        traj, x_np, s_np, _ = synth_inputs(cfg, 20260823)
        cases = [(traj, x_np, s_np, cfg["n"], cfg["g"])]
        workload = workload_text(cfg)
    ops = []
    for traj, x_np, s_np, n, g in cases:
        op = CpuSenseFp32(traj, n, g, cfg["width"], s_np, threads=threads)
        ops.append((op, op.forward(x_np)))
    times = []
    for k in range(args.warmup + args.steps):  # every step is one full solve
        op, y = ops[k % len(ops)]
        t0 = time.perf_counter()
        op.cg_sense(y, cfg["iters"], 1e-4)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    per = sum(times) / len(times)
    value = 1.0 / per
    return {
        "metric": METRIC, "impl": "reference", "value": round(value, 5), "unit": "recons/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(per * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload},
        "cpu_baseline": {"value": round(value, 5), "unit": "recons/s", "cores": threads, "kind": "port",
                         "sample": f"per step: one full {cfg['iters']}-iteration FP32 CG-SENSE solve of one case "
                                   f"({workload}) by the reference_sparse_solver fp32/fp32 CSR path restated "
                                   "(pinned to the reference's own output, tests/golden/solver_small.npz)"},
        "e2e": {"value": round(value, 5), "unit": "recons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def volume_bytes(plan, cfg: dict) -> dict:
    """Algorithmic (compulsory) bytes of each stage of one CG iteration of a volume plan."""
    n, g, c = cfg["n"], cfg["g"], cfg["c"]
    info = plan.info
    pix = n ** 3
    z1 = n * g * n * c * 8               # [i0][q2][i1][c] and [q2][i0][i1][c]
    z2 = g * g * n * c * 8               # [q2][q1][i0][c]
    panel_row = 8 * c
    m = plan.samples
    return {
        "fwd_rows": pix * 8 * 7 + c * pix * 8 + pix * 4 + z1,      # r, p, ap, x rw, smaps, scaling, z1
        "fwd_mid": z1 + z2,
        "fwd_cols": z2 + g ** 3 * panel_row,
        "interp_fwd": info["pack_bytes"][0] + g ** 3 * panel_row + m * panel_row,
        "interp_adj": info["pack_bytes"][1] + m * panel_row + info["active_rows"][1] * c * 8,
        "inv_cols": g ** 3 * c * 8 + z2,
        "inv_mid": z2 + z1,
        "inv_rows": z1 + c * pix * 8 + pix * 4 + pix * 8 * 3,       # z1, smaps, scaling, p, r, ap
        "cg_update": pix * 8 * 6,
    }


def run_volume(args, cfg) -> dict | None:
    """3D kooshball CG-SENSE: one volume plan (packed once, outside the timed region)."""
    import torch
    import torch.distributed as dist
    from oracle import nudft as onudft
    from trajsparsenufft_b200 import synth
    from trajsparsenufft_b200.operator import Plan

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900), device_id=dev)
    seed = 20260823 + rank
    n, g, c = cfg["n"], cfg["g"], cfg["c"]
    traj = synth.kooshball(cfg["spokes"], cfg["readout"])
    x_np = synth.ellipsoid_phantom(n, seed)
    s_np = synth.coil_maps3(n, c, seed)
    plan = Plan.from_trajectory(traj, im_size=n, grid_size=g, coils=c, width=cfg["width"], device=local)
    x_true = torch.from_numpy(x_np).to(dev)
    smaps = torch.from_numpy(s_np).to(dev)
    y_clean = plan.forward(x_true, smaps)
    # accuracy of the forward operator against the direct FP64 NUDFT on a sample subset
    sub = np.arange(0, plan.samples, plan.samples // 48)
    exact = onudft.Nudft3(traj[sub], n).forward(x_np, s_np)
    got = y_clean[:, torch.from_numpy(sub).to(dev)].cpu().numpy().astype(np.complex128)
    fwd_err = float(np.linalg.norm(got - exact) / np.linalg.norm(exact))
    gen = torch.Generator(device=dev).manual_seed(seed)
    rms = y_clean.abs().pow(2).mean().sqrt()
    noise = torch.complex(torch.randn(y_clean.shape, device=dev, generator=gen),
                          torch.randn(y_clean.shape, device=dev, generator=gen))
    y = (y_clean + noise * (1e-3 * rms / math.sqrt(2.0))).contiguous()
    del y_clean, noise
    x_out = torch.empty_like(x_true)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    iters, lam = cfg["iters"], 1e-4

    def step():
        plan.cg_sense(y, smaps, lam=lam, iters=iters, out=x_out, sync=False)

    _, hist, status = plan.cg_sense(y, smaps, lam=lam, iters=iters, out=x_out, sync=True)
    if not (status["positive_curvature"] and status["finite"]):
        raise RuntimeError(f"CG status {status}")
    recon_err = float(torch.linalg.vector_norm(x_out.abs() - x_true.abs()) / torch.linalg.vector_norm(x_true.abs()))
    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            starts[k].record()
            step()
            ends[k].record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    max_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in zip(starts, ends)), dev)
    value = job_rate(world, 1, args.steps, max_ms)

    # end to end with host buffers: y and maps in from pinned memory (next step's copy on a side
    # stream overlapping this step's solve), the volume back every step
    with NumaLocal(local):
        y_h = y.cpu().pin_memory()
        s_h = smaps.cpu().pin_memory()
        x_h = torch.empty(x_out.shape, dtype=x_out.dtype).pin_memory()
    y_d = [torch.empty_like(y) for _ in range(2)]
    s_d = [torch.empty_like(smaps) for _ in range(2)]
    main_s = torch.cuda.current_stream()
    side = torch.cuda.Stream(device=dev)
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def e2e_run(nsteps):
        copied = [ev() for _ in range(nsteps)]
        start, end = ev(), ev()
        start.record(main_s)
        side.wait_stream(main_s)
        with torch.cuda.stream(side):
            y_d[0].copy_(y_h, non_blocking=True)
            s_d[0].copy_(s_h, non_blocking=True)
            copied[0].record(side)
        for k in range(nsteps):
            b = k & 1
            main_s.wait_event(copied[k])
            if k + 1 < nsteps:
                side.wait_stream(main_s)
                with torch.cuda.stream(side):
                    y_d[b ^ 1].copy_(y_h, non_blocking=True)
                    s_d[b ^ 1].copy_(s_h, non_blocking=True)
                    copied[k + 1].record(side)
            plan.cg_sense(y_d[b], s_d[b], lam=lam, iters=iters, out=x_out, sync=False)
            x_h.copy_(x_out, non_blocking=True)
        end.record(main_s)
        torch.cuda.synchronize()
        return start.elapsed_time(end), None

    e2e_steps = max(3, args.steps // 4)
    e2e_run(2)
    e2e_ms, _, e2e_repeats = median_run(lambda: e2e_run(e2e_steps), dev)
    stages = plan.profile_stages(y, smaps, reps=5)
    alg = volume_bytes(plan, cfg)
    dominant = max(stages, key=stages.get)
    peak, peak_kind = measured_peaks()
    achieved = alg[dominant] / (stages[dominant] * 1e-3) / 1e9
    recon_bytes = solve_bytes(alg, iters, n ** 3 * 8, ("interp_adj", "inv_cols", "inv_mid", "inv_rows"))
    m = plan.samples
    out = {
        "metric": VOLUME_METRIC if cfg["n"] == 128 else VOLUME_METRIC.replace("128^3", f"{n}^3"), "value": round(value, 4), "unit": "recons/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f16x2->f32 (f64 CG scalars)", "data": "synthetic",
        "config": {"workload": f"{n}^3 volume, {g}^3 grid, {c} coils, golden-means kooshball {cfg['spokes']}x"
                               f"{cfg['readout']} ({m} samples/coil), KB J={cfg['width']}, {iters} CG iterations",
                   "recons_per_step": 1, "l2": "inputs larger than L2 (and a 256 MB flush between steps)",
                   "parallelism": f"replicas x{world}", "planner": "optimized (fast above 2048-column unions)",
                   "tiles": plan.info["tiles"], "groups": plan.info["groups"],
                   "pack_bytes": plan.info["pack_bytes"], "plan_seconds": round(plan.info["plan_seconds"], 1)},
        "accuracy": {"forward_rel_l2_vs_fp64_nudft": round(fwd_err, 6), "nudft_subsample": int(len(sub)),
                     "recon_magnitude_nrmse_vs_truth": round(recon_err, 5),
                     "residual_ratio": hist[-1] / hist[0]},
        "e2e": {"value": round(job_rate(world, 1, e2e_steps, e2e_ms), 4), "unit": "recons/s",
                "h2d_bytes_per_step": int(y.numel() * 8 + smaps.numel() * 8),
                "d2h_bytes_per_step": int(x_out.numel() * 8),
                "repeats": [round(job_rate(world, 1, e2e_steps, v), 4) for v in e2e_repeats],
                "statistic": f"median of {len(e2e_repeats)} runs of {e2e_steps} steps"},
        "gpu_launches": args.steps * (7 + 9 * iters + 3),
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1), "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                     "algorithmic_bytes_per_launch": alg[dominant], "launch_ms": round(stages[dominant], 5)},
        "step_roofline": {"algorithmic_bytes_per_recon": int(recon_bytes),
                          "achieved_GBs": round(recon_bytes * value / world / 1e9, 1),
                          "frac": round(recon_bytes * value / world / 1e9 / peak, 4)},
        "stage_ms": {k: round(v, 5) for k, v in stages.items()},
        "clocks": clocks.summary(),
        "cpu_baseline": None,
        "cpu_baseline_note": "the reference path is 2D only; no CPU volume path to time",
    }
    if world > 1:
        dist.destroy_process_group()
    return out if rank == 0 else None


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", choices=tuple(CONFIGS), default="headline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the batch48 / grad4 comparisons that follow the headline line's measurement")
    ap.add_argument("--interp", choices=("auto", "mma_sp", "tcgen05"), default="auto",
                    help="sparse interpolation kernel of the plans (headline configuration)")
    ap.add_argument("--streams", type=int, default=0, help="batch48: concurrent case streams (default 4)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    cfg = dict(CONFIGS[args.config])
    if args.streams > 0:
        cfg["streams"] = args.streams
    if args.impl == "reference":
        out = run_reference(args, cfg)
    elif cfg.get("batch"):
        out = run_batch(args, cfg)
    elif cfg.get("grad"):
        out = run_grad(args, cfg)
    elif cfg.get("volume"):
        out = run_volume(args, cfg)
    else:
        out = run_ours(args, cfg)
    if out is not None:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
