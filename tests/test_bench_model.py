"""bench.py's algorithmic-byte model of a CG solve (host arithmetic only)."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


class _Info:
    def __init__(self, pack_bytes, active_rows, samples):
        self.info = {"pack_bytes": pack_bytes, "active_rows": active_rows}
        self.samples = samples


def test_solve_bytes_counts_one_update_per_solve():
    cfg = {"n": 256, "g": 512, "c": 8}
    plan = _Info([27_406_848, 25_111_296], [131_072, 262_144], 131_072)
    alg = bench.algorithmic_bytes(plan, cfg)
    img = cfg["n"] ** 2 * 8
    rhs = ("interp_adj", "inv_cols", "inv_rows")
    per_iter = sum(v for k, v in alg.items() if k != "cg_update")
    # each extra iteration adds one fused iteration; cg_update is counted once per solve
    assert bench.solve_bytes(alg, 11, img, rhs) - bench.solve_bytes(alg, 10, img, rhs) == per_iter
    one = bench.solve_bytes(alg, 1, img, rhs)
    assert one == per_iter - 6 * img + alg["cg_update"] + sum(alg[k] for k in rhs)
    # the fused forward rows move 5 images more than the first (r in, p out) and the fused
    # inverse rows one image more than the last
    assert alg["fwd_rows"] - 5 * img > 0 and alg["inv_rows"] - img > 0


def test_volume_bytes_share_the_solve_model():
    cfg = {"n": 64, "g": 128, "c": 8}
    plan = _Info([137_000_000, 120_000_000], [2_000_000, 2_097_152], 262_144)
    alg = bench.volume_bytes(plan, cfg)
    assert {"fwd_mid", "inv_mid", "cg_update"} <= set(alg)
    img = cfg["n"] ** 3 * 8
    rhs = ("interp_adj", "inv_cols", "inv_mid", "inv_rows")
    per_iter = sum(v for k, v in alg.items() if k != "cg_update")
    assert bench.solve_bytes(alg, 10, img, rhs) == 10 * per_iter - 6 * img + alg["cg_update"] + sum(alg[k] for k in rhs)


def test_numa_local_is_a_no_op_without_nvml_answer():
    """bench.NumaLocal pins the allocating thread to the GPU's NUMA-local CPUs only when NVML
    names them; without a GPU it changes nothing and says so."""
    import os
    before = os.sched_getaffinity(0)
    with bench.NumaLocal(0) as numa:
        assert os.sched_getaffinity(0) == (numa.cpus or before)
    assert os.sched_getaffinity(0) == before
    info = numa.summary()
    assert info["allowed_cpus"] == len(before)
    assert info["pinned_on_gpu_node"] == bool(numa.cpus)
