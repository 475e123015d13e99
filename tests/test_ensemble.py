"""Batched ensemble: every realization of an ensemble step must equal, bit for bit, the same
realization run alone through its own handle with the same plan (the ensemble only schedules
the realizations' kernels together, as one CUDA graph per batch).  CPU tests cover the
standard ensemble's parameters and the split of realizations over GPUs, including a gloo
world-size-2 run of that split."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bastr_b200.ensemble import ensemble_configs, partition_by_cost, realization_cost


def test_standard_ensemble_parameters():
    cfgs = ensemble_configs()
    assert len(cfgs) == 96
    assert [c["ia"] for c in cfgs].count(256) == 32 and [c["ia"] for c in cfgs].count(1024) == 32
    assert sorted(c["seed"] for c in cfgs) == list(range(96))
    assert all(3 <= c["forcek"] <= 8 and 0.05 <= c["target_energy"] <= 0.1 for c in cfgs)
    assert all(c["forcemethod"] == 2 and c["precision"] == "fp32" for c in cfgs)
    assert ensemble_configs() == cfgs   # seeded: the same ensemble every time


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_covers_and_balances(world):
    cfgs = ensemble_configs()
    parts = partition_by_cost(cfgs, world)
    assert sorted(i for p in parts for i in p) == list(range(len(cfgs)))
    loads = [sum(realization_cost(cfgs[i]) for i in p) for p in parts]
    biggest = max(realization_cost(c) for c in cfgs)
    assert max(loads) - min(loads) <= biggest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    cfgs = ensemble_configs()
    mine = partition_by_cost(cfgs, world)[rank]
    # every rank computes the same split; gather each rank's indices and check the union
    t = torch.zeros(len(cfgs), dtype=torch.int64)
    t[mine] = rank + 1
    dist.all_reduce(t)
    q.put((rank, mine, t.tolist()))
    dist.destroy_process_group()


def test_partition_over_two_gloo_ranks():
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
    owner = res[0][2]
    assert owner == res[1][2]
    assert all(o in (1, 2) for o in owner)            # each realization owned by exactly one rank
    assert set(res[0][1]).isdisjoint(res[1][1])


# ---------------------------------------------------------------------------------------------
# GPU: ensemble against independent handles
# ---------------------------------------------------------------------------------------------
SMALL = [
    dict(ia=64, ja=64, ka=0, forcemethod=2, forcek=3, target_energy=0.06, lprojectd=True, deltat=1e-3, seed=0),
    dict(ia=64, ja=64, ka=0, forcemethod=2, forcek=5, target_energy=0.09, lprojectd=True, deltat=1e-3, seed=1),
    dict(ia=128, ja=128, ka=0, forcemethod=1, target_energy=1.0, deltat=2e-4, seed=2),
    dict(ia=16, ja=16, ka=16, forcemethod=1, target_energy=1.5, deltat=1e-3, seed=3),
]


def _field(c):
    from bastr_b200 import seeded_field
    return seeded_field(c["ia"], c["ja"], c.get("ka", 0), k0=3.0, seed=c["seed"])


def _alone(c, precision, nsteps, plan):
    from bastr_b200 import BastrGPU
    kw = {k: c[k] for k in ("forcemethod", "forcek", "target_energy", "lprojectd", "deltat") if k in c}
    with BastrGPU(c["ia"], c["ja"], c.get("ka", 0), precision=precision, **kw) as s:
        s.set_plan(plan)
        s.set_state(_field(c))
        recs = []
        for n in nsteps:
            recs += s.step(n)
        return recs, s.get_state()


def _same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


def _check_against_alone(ens, cfgs, precision, nsteps, got):
    plans = ens.plans()
    for i, c in enumerate(cfgs):
        recs, u = _alone(c, precision, nsteps, plans[i])
        g = [r for batch in got for r in batch[i]]
        for a, b in zip(g, recs):
            assert a.nstep == b.nstep and a.time == b.time
            assert _same([a.Esspe, a.Edspe, a.k2Edspe, a.kMEdspe, a.factor, a.E, *a.velgrad],
                         [b.Esspe, b.Edspe, b.k2Edspe, b.kMEdspe, b.factor, b.E, *b.velgrad]), (i, a, b)
        assert all(_same(x, y) for x, y in zip(ens.get_state(i), u)), i


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_ensemble_bitwise_equals_independent_runs(gpu_lib, precision):
    from bastr_b200 import BastrEnsemble
    cfgs = [dict(c, precision=precision) for c in SMALL]
    with BastrEnsemble(cfgs) as ens:
        for i, c in enumerate(cfgs):
            ens.set_state(i, _field(c))
        got = [ens.step(3), ens.step(2)]
        _check_against_alone(ens, cfgs, precision, (3, 2), got)


@pytest.mark.gpu
def test_ensemble_plans_and_tuner(gpu_lib):
    from bastr_b200 import BastrEnsemble
    cfgs = [dict(c, precision="fp64") for c in SMALL]
    with BastrEnsemble(cfgs) as ens:
        for i, c in enumerate(cfgs):
            ens.set_state(i, _field(c))
        ens.set_plan(2, i=1)
        ens.set_plan(1, i=3)
        assert ens.plans() == [0, 2, 0, 1]
        got = [ens.step(2)]
        _check_against_alone(ens, cfgs, "fp64", (2,), got)
    with BastrEnsemble(cfgs) as ens:
        for i, c in enumerate(cfgs):
            ens.set_state(i, _field(c))
        ms = ens.tune(nsteps=2, reps=1, max_share_log2=2)
        assert ms > 0 and all(0 <= p <= 2 for p in ens.plans())
        got = [ens.step(3)]   # the tuner restored the initial state
        _check_against_alone(ens, cfgs, "fp64", (3,), got)
