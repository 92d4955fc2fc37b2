"""The N > 1 path of bench.py (replicas, no collective on the data path) on
CPU: two gloo ranks agree on the job time (max over ranks) and solve
different images."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as tmp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        assert bench.dist_env() == (rank, rank, world)
        job_ms = bench.max_over_ranks(10.0 + 5.0 * rank, world)
        seed = bench.replica_seed(2, rank)
        from densecrf_ho_b200 import synth
        img = synth.make_image(16, 12, 21, seed)
        q.put((rank, job_ms, seed, int(img["rgb"].sum())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_replicas_max_over_ranks_gloo(world):
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert all(ms == 10.0 + 5.0 * (world - 1) for _, ms, _, _ in res)  # every rank sees the max
    assert len({seed for _, _, seed, _ in res}) == world               # distinct replica inputs
    assert len({h for _, _, _, h in res}) == world
