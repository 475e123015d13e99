"""Data-parallel closure training on CPU: two gloo ranks average their gradients with the same
call the NCCL ranks use before every Adam step, so every rank applies the same update."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch
    import torch.distributed as dist
    from bastr_b200.closure import average_gradient, nparams
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    g = torch.full((nparams(),), float(rank + 1)) + torch.arange(nparams(), dtype=torch.float32)
    average_gradient(g)
    q.put((rank, g[:3].tolist(), float(g.sum())))
    dist.destroy_process_group()


def test_gradient_average_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert res[0][1] == res[1][1] == [1.5, 2.5, 3.5]     # mean of rank 0 (1 + i) and rank 1 (2 + i)
    assert res[0][2] == res[1][2]
