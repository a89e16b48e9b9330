"""Per-trajectory autotuner: pick the planner settings whose packs interpolate fastest.

The pack-once step has free choices that do not change the operator, only how its nonzeros
are grouped into 16-row, K32 2:4 tiles: the row-grouping policy (trajectory order, Morton
order, overlap-greedy, packing256; nufft_layout_oracle.py:243-309) and the planner
(optimized / fast / search; export_torchkbnufft_gpu_case.py:46-99, :270-299).  The
reference ranks such variants offline (run_case / metric_rank, nufft_layout_oracle.py:638-689)
by packing metrics; here every candidate is planned, its forward and adjoint sparse
interpolation launches are timed on the GPU (CUDA events, tsn_profile_stages), and the
fastest is kept.  Choices are cached per trajectory in a JSON file keyed by a SHA-256 of the
trajectory samples, the plan shape and the device name, so a trajectory is tuned once.

    plan, choice = autotune.plan(trajectory, im_size=256, grid_size=512, coils=8)
"""

from __future__ import annotations

import hashlib
import json
import os
import time
from pathlib import Path

import numpy as np

DEFAULT_CANDIDATES = (("optimized", "morton"), ("optimized", "overlap"), ("optimized", "trajectory"),
                      ("optimized", "packing256"))


def cache_path() -> Path:
    """$TSN_AUTOTUNE_CACHE, else ~/.cache/trajsparsenufft_b200/autotune.json."""
    env = os.environ.get("TSN_AUTOTUNE_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "trajsparsenufft_b200" / "autotune.json"


def trajectory_key(trajectory, im_size: int, grid_size: int, coils: int, width: int, device_name: str = "") -> str:
    """SHA-256 of the float32 trajectory and the plan shape; [M, 3] (volume) trajectories add a
    dimension tag, so an image and a volume trajectory with the same bytes never share a key."""
    a = np.asarray(trajectory, dtype=np.float32)
    dims = 3 if a.ndim == 2 and a.shape[1] == 3 else 2
    t = np.ascontiguousarray(a.reshape(-1, dims))
    h = hashlib.sha256()
    h.update(t.tobytes())
    h.update(f"|{im_size}|{grid_size}|{coils}|{width}|{device_name}".encode())
    if dims == 3:
        h.update(b"|3d")
    return h.hexdigest()


def _load(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _store(path: Path, key: str, entry: dict) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    data = _load(path)
    data[key] = entry
    tmp = path.with_suffix(path.suffix + f".{os.getpid()}.tmp")
    tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
    tmp.replace(path)  # atomic on POSIX: concurrent tuners never leave a torn file


def interp_ms(plan, reps: int = 10) -> float:
    """Forward + adjoint interpolation time per CG iteration of a plan (ms, CUDA events)."""
    import torch
    c = plan.coils
    dev = torch.device("cuda", torch.cuda.current_device())
    y = torch.randn(c, plan.samples, dtype=torch.complex64, device=dev)
    smaps = torch.ones(plan.maps_shape, dtype=torch.complex64, device=dev) / np.sqrt(c)
    st = plan.profile_stages(y, smaps, reps=reps)
    return st["interp_fwd"] + st["interp_adj"]


def choose(key: str, candidates, build, measure, cache: Path | None = None) -> tuple[object, dict]:
    """Build each candidate, measure it, keep the fastest; reuse a cached choice.

    build(planner, policy) -> plan; measure(plan) -> ms.  Returns (plan, choice entry)."""
    if cache is not None:
        hit = _load(cache).get(key)
        if hit and (hit["planner"], hit["policy"]) in {tuple(c) for c in candidates}:
            return build(hit["planner"], hit["policy"]), dict(hit, cached=True)
    best, best_entry, trials = None, None, []
    for planner, policy in candidates:
        t0 = time.perf_counter()
        plan = build(planner, policy)
        plan_s = time.perf_counter() - t0
        ms = float(measure(plan))
        trials.append({"planner": planner, "policy": policy, "interp_ms": ms, "plan_seconds": round(plan_s, 3)})
        if best_entry is None or ms < best_entry["interp_ms"]:
            if best is not None:
                best.close()
            best, best_entry = plan, trials[-1]
        else:
            plan.close()
    entry = {"planner": best_entry["planner"], "policy": best_entry["policy"], "interp_ms": best_entry["interp_ms"],
             "trials": trials}
    if cache is not None:
        _store(cache, key, entry)
    return best, dict(entry, cached=False)


def plan(trajectory, *, im_size=256, grid_size=512, coils=8, width=6, candidates=DEFAULT_CANDIDATES,
         cache: bool | str | Path = True, device=None, reps: int = 10):
    """Autotuned Plan for a trajectory: (plan, choice) with the chosen planner / policy."""
    import torch

    from .operator import Plan
    dev = torch.cuda.current_device() if device is None else int(device)
    name = torch.cuda.get_device_name(dev)
    key = trajectory_key(trajectory, im_size, grid_size, coils, width, name)
    path = None if cache is False else (cache_path() if cache is True else Path(cache))

    def build(planner, policy):
        return Plan.from_trajectory(trajectory, im_size=im_size, grid_size=grid_size, coils=coils, width=width,
                                    planner=planner, policy=policy, device=dev)

    with torch.cuda.device(dev):
        return choose(key, candidates, build, lambda p: interp_ms(p, reps), path)
