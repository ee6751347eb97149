"""Host side of the multi-GPU paths, on CPU: the job split over ranks and the timing
reduction (gloo, world size 2), and that only rank 0 of the reference arm works or prints."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_shard_jobs_covers_every_job_once_and_balances():
    from pic_cuda_b200.shard import shard_jobs
    rng = np.random.default_rng(3)
    work = rng.uniform(1.0, 100.0, 257)
    for world in (1, 2, 3, 8):
        parts = shard_jobs(work, world)
        assert len(parts) == world
        flat = sorted(j for p in parts for j in p)
        assert flat == list(range(len(work)))
        loads = [work[p].sum() for p in parts]
        # largest-first greedy: no rank exceeds the mean by more than the largest job
        assert max(loads) <= sum(loads) / world + work.max() + 1e-9
    assert shard_jobs(work, 4) == shard_jobs(list(work), 4)   # same split on every rank
    assert shard_jobs([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard_jobs(work, 0)


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from pic_cuda_b200.shard import reduce_timing
    ms, work = reduce_timing(10.0 + rank, 100.0 * (rank + 1), dist)
    q.put((rank, ms, work))
    dist.barrier()
    dist.destroy_process_group()


def test_reduce_timing_gloo_world_2():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 11.0, 300.0), (1, 11.0, 300.0)]


def test_reduce_timing_single_rank_is_identity():
    from pic_cuda_b200.shard import reduce_timing
    assert reduce_timing(3.5, 7.0, None) == (3.5, 7.0)


def test_reference_arm_only_rank0_works():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_shard_requests_round_robin_in_arrival_order():
    from pic_cuda_b200.shard import shard_requests
    rng = np.random.default_rng(5)
    arr = list(rng.exponential(1.0, 101).cumsum())
    arr[7] = arr[8]   # a tie, broken by index
    parts = [shard_requests(arr, 3, r) for r in range(3)]
    assert sorted(k for p in parts for k in p) == list(range(101))
    order = sorted(range(101), key=lambda k: (arr[k], k))
    assert parts[1] == order[1::3]
    for p in parts:
        assert all(arr[a] <= arr[b] for a, b in zip(p, p[1:]))
    with pytest.raises(ValueError):
        shard_requests(arr, 2, 2)


def _gather_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from pic_cuda_b200.shard import gather_latencies
    q.put((rank, gather_latencies([float(rank)] * (rank + 1), dist)))
    dist.barrier()
    dist.destroy_process_group()


def test_gather_latencies_gloo_world_2():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gather_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, [0.0, 1.0, 1.0]), (1, [0.0, 1.0, 1.0])]
