"""The N > 1 harness on CPU: two gloo ranks reduce step times (max) and rows (sum)."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from polars_b200.replicas import barrier, dist_env, reduce_step_stats

    assert dist_env() == (rank, rank, world)
    barrier()
    ms, rows = reduce_step_stats(1.0 + rank, 100 * (rank + 1))
    q.put((rank, ms, rows))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2.0, 300), (1, 2.0, 300)]


def test_single_process_is_identity():
    from polars_b200.replicas import reduce_step_stats

    assert reduce_step_stats(3.5, 7) == (3.5, 7)
