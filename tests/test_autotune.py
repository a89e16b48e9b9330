"""Autotuner selection and per-trajectory cache (CPU: fake plans and timings; GPU: a real plan)."""
import json

import numpy as np
import pytest

from trajsparsenufft_b200 import autotune, synth


class _FakePlan:
    closed = 0

    def __init__(self, planner, policy):
        self.planner, self.policy = planner, policy

    def close(self):
        _FakePlan.closed += 1


def test_choose_keeps_fastest_and_caches(tmp_path):
    times = {("optimized", "morton"): 3.0, ("optimized", "overlap"): 2.0, ("fast", "trajectory"): 5.0}
    built, measured = [], []

    def build(pl, po):
        built.append((pl, po))
        return _FakePlan(pl, po)

    def measure(p):
        measured.append((p.planner, p.policy))
        return times[(p.planner, p.policy)]

    cache = tmp_path / "tune.json"
    plan, choice = autotune.choose("k1", list(times), build, measure, cache)
    assert (plan.planner, plan.policy) == ("optimized", "overlap") and not choice["cached"]
    assert len(choice["trials"]) == 3 and _FakePlan.closed >= 2
    entry = json.loads(cache.read_text())["k1"]
    assert entry["policy"] == "overlap" and entry["interp_ms"] == 2.0
    built.clear(), measured.clear()
    plan2, choice2 = autotune.choose("k1", list(times), build, measure, cache)
    assert choice2["cached"] and built == [("optimized", "overlap")] and measured == []
    # a cached choice outside the candidate list is re-tuned
    plan3, choice3 = autotune.choose("k1", [("fast", "trajectory")], build, measure, cache)
    assert not choice3["cached"] and plan3.policy == "trajectory"


def test_trajectory_key_is_stable_and_shape_sensitive():
    t = synth.golden_radial(8, 64)
    k = autotune.trajectory_key(t, 64, 128, 4, 6, "dev")
    assert k == autotune.trajectory_key(t.astype(np.float64), 64, 128, 4, 6, "dev")
    assert k != autotune.trajectory_key(t, 64, 128, 8, 6, "dev")
    assert k != autotune.trajectory_key(t[:-1], 64, 128, 4, 6, "dev")


def test_volume_trajectory_key():
    v = synth.kooshball(7, 9)                      # 63 samples: 189 values, not a multiple of 2
    k = autotune.trajectory_key(v, 64, 128, 4, 4, "dev")
    assert k == autotune.trajectory_key(v.astype(np.float64), 64, 128, 4, 4, "dev")
    flat = v.reshape(-1)[:126].reshape(-1, 2)       # the same leading bytes as an image trajectory
    assert k != autotune.trajectory_key(flat, 64, 128, 4, 4, "dev")


@pytest.mark.gpu
def test_autotuned_plan_on_gpu(tmp_path):
    pytest.importorskip("torch")
    import sys
    sys.path.insert(0, str(__import__("pathlib").Path(__file__).parent))
    from gpu_cases import case
    traj, x, s, n, g, c, j, _ = case("small")
    cands = [("optimized", "morton"), ("optimized", "trajectory")]
    plan, choice = autotune.plan(traj, im_size=n, grid_size=g, coils=c, width=j, candidates=cands,
                                 cache=tmp_path / "t.json")
    assert (choice["planner"], choice["policy"]) in cands and not choice["cached"]
    assert choice["interp_ms"] == min(t["interp_ms"] for t in choice["trials"])
    plan2, choice2 = autotune.plan(traj, im_size=n, grid_size=g, coils=c, width=j, candidates=cands,
                                   cache=tmp_path / "t.json")
    assert choice2["cached"] and choice2["policy"] == choice["policy"]
    assert plan2.info["tiles"] == plan.info["tiles"]


@pytest.mark.gpu
def test_autotuned_volume_plan_on_gpu(tmp_path):
    pytest.importorskip("torch")
    import sys
    sys.path.insert(0, str(__import__("pathlib").Path(__file__).parent))
    from gpu_cases import volume_case
    traj, x, s, n, g, c, j = volume_case("vol64")
    cands = [("optimized", "morton"), ("optimized", "trajectory")]
    plan, choice = autotune.plan(traj, im_size=n, grid_size=g, coils=c, width=j, candidates=cands,
                                 cache=tmp_path / "v.json")
    assert plan.dims == 3 and (choice["planner"], choice["policy"]) in cands and not choice["cached"]
    assert choice["interp_ms"] == min(t["interp_ms"] for t in choice["trials"]) > 0
    _, choice2 = autotune.plan(traj, im_size=n, grid_size=g, coils=c, width=j, candidates=cands,
                               cache=tmp_path / "v.json")
    assert choice2["cached"] and choice2["policy"] == choice["policy"]
