"""The multi-GPU bench path on CPU: two gloo ranks take the barrier and the max of their
device times exactly as the NCCL ranks of ``bench.py --gpus N`` do, and the whole-job value is
the sum of the replicas' steps over the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    ctx = bench.DistCtx("gloo")
    ctx.barrier()
    ms = ctx.max(10.0 * (rank + 1))            # rank r "took" 10(r+1) ms for its steps
    v = bench.whole_job_value(100, ms, world)
    ctx.barrier()
    ctx.close()
    q.put((rank, ms, v))


@pytest.mark.parametrize("world", [2])
def test_replicas_max_over_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    out = sorted(q.get(timeout=5) for _ in range(world))
    slowest = 10.0 * world
    for rank, ms, v in out:
        assert ms == slowest
        assert v == pytest.approx(world * 100 / (slowest * 1e-3))
