"""Multi-GPU host logic on CPU: two gloo ranks shard the twist batch with no data
exchange (each rank owns its own twists) and time the job as the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    tw = bench.twists(5, rank=rank)
    systems = bench.build_systems(tw)
    # a stand-in for this rank's device time: ranks differ, the job time is the max
    local = [10.0 * (rank + 1), 1.0 + rank]
    red = bench.reduce_max(local)
    out.put((rank, tw.tolist(), [s[0] for s in systems], [len(s[3]) for s in systems], red))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_and_max_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=120)
        res[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    tw0, tw1 = np.array(res[0][1]), np.array(res[1][1])
    assert not np.any(np.all(np.isclose(tw0[:, None, :], tw1[None, :, :]), axis=-1))  # disjoint twists
    for r in (0, 1):
        assert res[r][2] == [27] * 5 and res[r][3] == [485] * 5
        assert res[r][4] == [20.0, 2.0]  # both ranks see the max
