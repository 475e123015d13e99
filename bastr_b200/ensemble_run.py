"""Multi-rank runner of the batched ensemble: one process per GPU (torchrun), realizations split by
cost over the ranks, no data exchanged on the data path.

    python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 \\
        -m bastr_b200.ensemble_run [--steps 1000] [--batch 10] [--n-per-size 32]

Every rank computes the same split (``partition_by_cost``: longest first by N log N), builds a
``BastrEnsemble`` of its share on its own GPU, sets each realization's seeded field, advances all
of them with ``BastrEnsemble.run`` (one CUDA-graph replay per batch, device-timed), and reports
per realization its final record.  Rank 0 gathers the reports (``gather_object``) in the original
realization order and the slowest rank's device time (all-reduce MAX): the job's throughput is
the realization-steps of all ranks over that time.  The reference runs one field per MPI job
(parallel.F90:128-173 sets up the communicator it would use); realizations are independent, so
the only collectives are this final gather and the timing reduction.
"""
from __future__ import annotations

import argparse
import json
import os

from .ensemble import ensemble_configs, partition_by_cost


def _default_field(cfg):
    from .initfield import seeded_field
    return seeded_field(cfg["ia"], cfg["ja"], cfg.get("ka", 0), k0=cfg.get("k0", 4.0), seed=cfg["seed"])


def _default_ensemble(configs, device):
    from .ensemble import BastrEnsemble
    return BastrEnsemble(configs, device=device)


def run_sharded(configs, nsteps: int, batch: int = 10, dist=None, device: int = 0,
                make_ensemble=_default_ensemble, make_field=_default_field) -> dict | None:
    """Runs this rank's share of the ensemble; returns the gathered summary on rank 0 (None on the
    other ranks).  `dist`: torch.distributed with an initialised process group, or None for one
    rank.  `make_ensemble(configs, device)` and `make_field(cfg)` build the ensemble and the
    initial fields (the defaults use the library and the seeded generator)."""
    rank = dist.get_rank() if dist else 0
    world = dist.get_world_size() if dist else 1
    parts = partition_by_cost(configs, world)
    mine = parts[rank]
    reports = []
    ms = 0.0
    if mine:
        ens = make_ensemble([configs[i] for i in mine], device)
        try:
            for j, i in enumerate(mine):
                ens.set_state(j, make_field(configs[i]))
            ms = ens.run(nsteps, batch)
            recs = ens.step(1)   # the next step's record: diagnostics of the advanced state
            for j, i in enumerate(mine):
                r = recs[j][0]
                reports.append({"index": i, "rank": rank, "nstep": int(r.nstep), "Esspe": r.Esspe, "Edspe": r.Edspe})
        finally:
            ens.close()
    if dist:
        import torch
        t = torch.tensor([ms], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(reports, gathered, dst=0)
    else:
        ms_max, gathered = ms, [reports]
    if rank != 0:
        return None
    by_index = sorted((r for part in gathered for r in part), key=lambda r: r["index"])
    steps_total = nsteps * len(configs)
    return {"realizations": len(configs), "ranks": world, "steps": nsteps, "device_ms_max": ms_max,
            "realization_steps_per_s": steps_total / (ms_max * 1e-3) if ms_max > 0 else None,
            "partition": parts, "reports": by_index}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--batch", type=int, default=10)
    ap.add_argument("--n-per-size", type=int, default=32)
    args = ap.parse_args()
    import datetime

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    out = run_sharded(ensemble_configs(args.n_per_size), args.steps, args.batch,
                      dist=dist if world > 1 else None, device=local)
    if world > 1:
        dist.destroy_process_group()
    if out is not None:
        out.pop("reports")
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
