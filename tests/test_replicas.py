"""Multi-GPU plan: replicas only.  Scenes are independent, so `bench.py --gpus N` runs one
replica per rank on its own scenes with no collective on the data path; the only
collectives are the timing reduction (max over ranks) and barriers.  This checks that host
logic with two gloo ranks on the CPU: distinct scene sets per rank, the max-over-ranks
time and the whole-job throughput agree on every rank.
"""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    targets = bench.scene_node_targets(64, bench.rank_seed(2, rank)).tolist()
    local_ms = 100.0 + 25.0 * rank                 # a slower second rank
    max_ms = bench.max_over_ranks(local_ms, world, "cpu")
    value = bench.job_throughput(world, 64, 20, max_ms)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, targets, max_ms, value))


def test_two_replicas_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, m0, v0), (r1, t1, m1, v1) = res
    assert t0 != t1                      # each replica solves its own scenes
    assert m0 == m1 == 125.0             # the slowest rank's time on every rank
    assert v0 == v1 == pytest.approx(2 * 64 * 20 / 0.125)
