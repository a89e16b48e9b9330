"""Multi-GPU replica bookkeeping of bench.py on CPU (world_size 2, gloo).

The path shards by reconstruction with no data exchange: every rank solves its own cases
and the job time is the max over ranks.  These ranks run bench.py's aggregation helpers over
a real gloo process group and check the max-over-ranks time, the whole-job rate and that
ranks draw disjoint case seeds.
"""
import datetime
import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")

ROOT = Path(__file__).resolve().parents[1]
RANK_MS = [12.5, 17.0]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, str(ROOT))
    import bench
    from trajsparsenufft_b200 import synth
    max_ms = bench.max_over_ranks(RANK_MS[rank], torch.device("cpu"))
    rate = bench.job_rate(world, 48, 10, max_ms)
    seeds = [c["seed"] for c in synth.uneven_batch(4, 20260823 + 1000 * rank)]
    dist.barrier()
    q.put((rank, max_ms, rate, seeds))
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_replicas_take_the_max_over_ranks():
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in results] == [max(RANK_MS)] * 2
    assert all(abs(r[2] - 2 * 48 * 10 / (max(RANK_MS) / 1e3)) < 1e-9 for r in results)
    assert not set(results[0][3]) & set(results[1][3])


def test_single_process_aggregation_is_local():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5, torch.device("cpu")) == 3.5
    assert bench.job_rate(1, 1, 100, 86.8) == pytest.approx(1152.07, rel=1e-4)
