"""The N > 1 path of bench.py on CPU: two gloo ranks run the replica
aggregation (barrier, max over ranks of the step time, whole-job rate) and
the reference arm's rank rule (only rank 0 reports)."""
from __future__ import annotations

import os
import sys

import pytest
import torch.multiprocessing as mp


def _rank_main(rank: int, world: int, port: int, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench._barrier(world)
        # rank r "took" 2 + r ms for 1,000 units: the job is as slow as rank 1
        rate, ms = bench.replica_rate(world, 1000.0, 2.0 + rank)
        # one job split over the ranks: rank r did 100 * (r + 1) units
        prate, pms = bench.partition_rate(world, 100.0 * (rank + 1), 2.0 + rank)
        args = type("A", (), {"steps": 1, "warmup": 0, "workload": "plain"})()
        ref = bench.run_reference(args) if rank != 0 else "rank0"
        out.put((rank, rate, ms, ref, prate, pms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_the_driver():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, rate, ms, ref, prate, pms in res:
        assert ms == pytest.approx(3.0)                     # max over ranks
        assert rate == pytest.approx(2000.0 / 3.0e-3)       # all units / slowest time
        assert pms == pytest.approx(3.0) and prate == pytest.approx(300.0 / 3.0e-3)
    assert res[1][3] is None                                # rank 1 of the reference arm prints nothing


def test_lpt_partition_packs_scenes_by_triangles():
    """The batch's longest-processing-time packing: every scene on exactly
    one rank, each rank's load within the LPT bound (4/3 of the optimum, so
    within the largest scene of the mean), the same packing on every rank."""
    import numpy as np

    from p2cccd_b200.batch import lpt_partition

    rng = np.random.default_rng(0)
    w = np.exp(rng.uniform(np.log(1e3), np.log(2e5), 256))
    for n in (1, 2, 3, 8):
        bins = lpt_partition(w, n)
        flat = sorted(i for b in bins for i in b)
        assert flat == list(range(256))
        loads = [w[b].sum() for b in bins]
        assert max(loads) <= w.sum() / n + w.max() + 1e-6
        assert max(loads) <= 4.0 / 3.0 * max(w.sum() / n, w.max()) + 1e-6
        assert lpt_partition(w, n) == bins
    with pytest.raises(ValueError):
        lpt_partition(w, 0)
