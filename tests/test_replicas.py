"""bench.py --gpus N runs N replicas: every rank proves its own shard (its own
seeded workload), the only collective is the MAX of the timed intervals, and
the whole-job value counts every rank's steps.  Two gloo ranks on the CPU."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import datetime
    import types

    import numpy as np
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        args = types.SimpleNamespace(ell=12, workload="memory", chunk=32)
        wl = bench.Workload(args, rank, 3)
        digest = int(np.bitwise_xor.reduce(wl.zs[0].astype(np.uint64))) ^ int(wl.pp[0, 0, 0])
        ms = 100.0 + 50.0 * rank                     # this rank's timed interval
        slowest = bench.max_over_ranks(ms, dist)
        value = bench.replica_value(world, 5, slowest)
        seen = [None] * world
        dist.all_gather_object(seen, digest)         # test only: compare the ranks' workloads
        q.put((rank, slowest, value, seen))
    finally:
        dist.destroy_process_group()


def test_two_replicas_own_workloads_and_max_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for rank, slowest, value, seen in out:
        assert slowest == 150.0                      # both ranks report the slowest rank
        assert abs(value - 2 * 5 / 0.150) < 1e-9     # whole-job steps over the slowest time
        assert seen[0] != seen[1]                    # each rank proves its own shard
