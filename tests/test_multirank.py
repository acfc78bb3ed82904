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


def _stub_main(argv):
    """bench.main with a CPU stand-in for the GPU work of a rank (rank r takes r+1 times as
    long), so the rank logic around it -- rendezvous, max over ranks, rank 0's line -- runs
    as it does on GPUs."""
    import bench

    def fake_run_gpu(args, rank, world):
        ms = 100.0 * (rank + 1) * args.steps
        value, e_max, e2e_value = bench.job_rates(args, world, ms, 50.0 * (rank + 1))
        systems = bench.build_systems(bench.twists(args.twists, rank=rank))
        return {"value": value, "ms_per_step": e_max / args.steps, "e2e_value": e2e_value, "h2d": 1, "d2h": 2,
                "niter_mean": 12.0, "niter_min": 12, "niter_max": 12, "fails": 0, "rc": 0,
                "stats": {"k_update": (1.0, 10)}, "clocks": {}, "ring_threads": [32], "fp64_peak": 37.0,
                "e2e_stage_ms": {}, "e2e_runs_ms": [], "ecorr_first": -2.2, "e2_first": -2.4,
                "launches_per_step": 100, "systems": systems, "replay_niter_mean": 33.0,
                "replay_vs_diis_max_dE": 0.0, "other": None}

    bench.run_gpu = fake_run_gpu
    bench.main(argv)


def test_bench_launches_its_own_ranks_and_reports_the_slowest():
    """`bench.py --gpus 2` without torchrun starts two ranks itself; rank 0 alone prints the
    line, whose rate is the whole job's: 2 ranks x twists x steps over the slower rank's time."""
    import json
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    here = os.path.dirname(os.path.abspath(__file__))
    argv = ["--gpus", "2", "--steps", "3", "--warmup", "3", "--twists", "2", "--no-cpu-baseline",
            "--serve-requests", "0"]
    code = ("import sys; sys.path[:0] = [%r, %r]; import bench, test_multirank as t; "
            "sys.exit(bench.launch_ranks(2, t._stub_main, %r))" % (root, here, argv))
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["scaling"] == "weak"
    # the slower rank took 200 ms per step: 2 ranks x 2 twists per 0.2 s
    assert abs(line["value"] - 2 * 2 / 0.2) < 1e-9
    assert abs(line["ms_per_step"] - 200.0) < 1e-9
    assert abs(line["e2e"]["value"] - 2 * 2 / 0.1) < 1e-9
