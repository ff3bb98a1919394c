"""The N > 1 path of bench.py on CPU: two ranks over gloo (127.0.0.1).
The sub-swath pairs are replicas -- each rank its own seeded scene, no
exchange on the data path -- so the only collective is the max over ranks of
the step time; the whole-job value counts every rank's pairs over the
slowest rank's time, and the reference arm runs on rank 0 alone."""
import os
import socket
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank                      # rank 1 is the slow one
        ms_max = bench.max_over_ranks(ms, dist, world, "cpu")
        seed = bench.rank_config(bench.CONFIGS["subswath"], rank)["seed"]
        q.put((rank, ms_max, seed, bench.whole_job_value(world, 9, ms_max)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_over_ranks_and_replica_seeds():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [o[1] for o in out] == [15.0, 15.0]          # both ranks see the slowest time
    assert out[0][2] != out[1][2]                       # each rank its own scene
    assert out[0][3] == out[1][3] == pytest.approx(2 * 9 * 1e3 / 15.0)


def test_reference_arm_runs_on_rank_zero_only():
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        config = "subswath"
        steps = warmup = 1
    # rank 1 returns at once: no scene, no work, no output
    assert bench.run_reference(Args(), 1, 2) is None
