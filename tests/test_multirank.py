"""The multi-GPU path of bench.py on CPU: replicas only, so its one collective is the
max-over-ranks of the timings (gloo ranks here; NCCL under torchrun on GPUs)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.max_over_ranks([10.0 + rank, 5.0 - rank, 1.5 * (rank + 1)], dist, device="cpu")
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_max_over_ranks_gloo(world):
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        assert results[r] == [10.0 + world - 1, 5.0, 1.5 * world]


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([1, 2.5], None) == [1.0, 2.5]
