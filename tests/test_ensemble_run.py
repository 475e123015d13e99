"""The multi-rank ensemble runner on CPU: two gloo ranks split the 96 standard realizations by
cost, each "runs" its share through a stand-in ensemble (no GPU: the step is replaced by a
deterministic function of the configuration), and rank 0 gathers every realization exactly once,
in order, with the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _Rec:
    def __init__(self, nstep, es, ed):
        self.nstep, self.Esspe, self.Edspe = nstep, es, ed


class _FakeEnsemble:
    """Stand-in for BastrEnsemble: records derived from each realization's seed and size."""

    def __init__(self, configs, device):
        self.configs = configs
        self.n = len(configs)
        self.nstep = 0
        self.fields = [None] * self.n

    def set_state(self, i, u):
        self.fields[i] = u

    def run(self, nsteps, batch):
        assert nsteps % batch == 0
        self.nstep += nsteps
        # device time proportional to this rank's cost, as the real graph replays would be
        return 1e-6 * sum(c["ia"] * c["ja"] for c in self.configs)

    def step(self, n):
        return [[_Rec(self.nstep, float(c["seed"]), float(c["ia"]))] for c in self.configs]

    def close(self):
        pass


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist

    from bastr_b200.ensemble import ensemble_configs
    from bastr_b200.ensemble_run import run_sharded
    dist.init_process_group("gloo")
    cfgs = ensemble_configs()
    out = run_sharded(cfgs, 40, batch=10, dist=dist, make_ensemble=_FakeEnsemble,
                      make_field=lambda c: ("field", c["seed"]))
    dist.destroy_process_group()
    q.put((rank, out))


def test_sharded_ensemble_gathers_every_realization_once():
    from bastr_b200.ensemble import ensemble_configs, partition_by_cost
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    res = dict(q.get(timeout=5) for _ in range(world))
    assert res[1] is None
    out = res[0]
    cfgs = ensemble_configs()
    parts = partition_by_cost(cfgs, world)
    assert out["partition"] == parts and out["ranks"] == world
    reps = out["reports"]
    assert [r["index"] for r in reps] == list(range(len(cfgs)))
    for r in reps:
        assert r["Esspe"] == cfgs[r["index"]]["seed"] and r["nstep"] == 40
        assert r["index"] in parts[r["rank"]]
    slowest = max(1e-6 * sum(cfgs[i]["ia"] * cfgs[i]["ja"] for i in p) for p in parts)
    assert out["device_ms_max"] == pytest.approx(slowest)
    assert out["realization_steps_per_s"] == pytest.approx(40 * len(cfgs) / (slowest * 1e-3))
