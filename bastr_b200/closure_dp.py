"""Data-parallel training of the learned closure over ranks: one process per GPU (torchrun).

    python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 \\
        -m bastr_b200.closure_dp [--fine 256] [--ratio 4] [--train-seeds 0 1 2 3 4 5 6 7] \\
        [--spinup 400] [--every 100] [--snapshots 4] [--iters 2000] [--out weights.npy]

1. Data, sharded: the training seeds are dealt out round-robin; each rank advances its seeds as
   one ensemble of fine realizations on its own GPU (CUDA-graph replays) and forms every
   snapshot's filtered field and subgrid term there (bastr_ensemble_subgrid).  No field crosses
   between ranks.
2. The targets' scale tau_rms is global: one all-reduce of (sum of squares, count).
3. Training: every rank holds the same initial weights; before each Adam step the gradient is
   averaged over the ranks (one all-reduce of the 4835 floats, `average_gradient`), so the ranks'
   weights stay identical.  Rank 0 writes the FP32 weights and a JSON summary.

Collectives: the scale all-reduce, one gradient all-reduce per step, a final MAX of the device
times.  The reference has no closure; this is the multi-GPU form of its training.
"""
from __future__ import annotations

import argparse
import json
import os


def shard_seeds(seeds, rank: int, world: int):
    """Round-robin share of the training seeds (every rank computes the same split)."""
    return list(seeds[rank::world])


def make_pairs(seeds, args, device: int = 0):
    """This rank's (ub, tau) pairs from its seeds, made by the batched solver on its GPU."""
    from . import BastrEnsemble, seeded_field
    nf = args.fine
    phys = dict(reynolds=args.reynolds, deltat=args.dt, forcemethod=1, target_energy=args.target)
    cfgs = [dict(ia=nf, ja=nf, ka=nf, precision="fp32", velgrad_every=0, kmax=nf // 3, seed=sd, **phys)
            for sd in seeds]
    pairs = []
    ms = 0.0
    if not cfgs:
        return pairs, ms
    with BastrEnsemble(cfgs, device=device) as ens:
        for i, sd in enumerate(seeds):
            ens.set_state(i, seeded_field(nf, nf, nf, k0=args.k0, seed=sd))
        ms += ens.run(args.spinup, args.batch)
        for _ in range(args.snapshots):
            ms += ens.run(args.every, args.batch)
            pairs += [ens.subgrid(i, args.ratio) for i in range(len(cfgs))]
    return pairs, ms


def global_tau_rms(pairs, group, device):
    """sqrt(mean(tau^2)) over every rank's targets (one all-reduce of two numbers)."""
    import torch
    import torch.distributed as dist
    s = torch.zeros(2, dtype=torch.float64, device=device)
    for _, t in pairs:
        s[0] += torch.sum(t.double() ** 2)
        s[1] += t.numel()
    if group is not None and dist.get_world_size(group) > 1:
        dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
    return float(torch.sqrt(s[0] / s[1]).item())


def train_dp(net, pairs, iters: int, lr: float, group=None):
    """Scales this rank's targets by the global tau_rms and trains `net` data parallel; returns
    (tau_rms, loss history of this rank's pairs)."""
    dev = pairs[0][1].device
    tau_rms = global_tau_rms(pairs, group, dev)
    train = [(ub.contiguous(), (t / tau_rms).contiguous()) for ub, t in pairs]
    hist = net.train(train, iters=iters, lr=lr, group=group)
    return tau_rms, hist


def main():
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    from .closure import Net

    ap = argparse.ArgumentParser()
    ap.add_argument("--fine", type=int, default=256)
    ap.add_argument("--ratio", type=int, default=4)
    ap.add_argument("--reynolds", type=float, default=40.0)
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--target", type=float, default=1.5)
    ap.add_argument("--k0", type=float, default=3.0)
    ap.add_argument("--train-seeds", type=int, nargs="+", default=list(range(8)))
    ap.add_argument("--spinup", type=int, default=400)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--snapshots", type=int, default=4)
    ap.add_argument("--batch", type=int, default=10)
    ap.add_argument("--iters", type=int, default=2000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--net-seed", type=int, default=0)
    ap.add_argument("--out", default="closure_weights.npy")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", 1))
    rank = int(os.environ.get("RANK", 0))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if world > len(args.train_seeds):
        # the same test on every rank, before any collective: no rank is left waiting
        raise SystemExit(f"{world} ranks need at least {world} training seeds, got {len(args.train_seeds)}")
    torch.cuda.set_device(local)
    group = None
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        group = dist.group.WORLD
    seeds = shard_seeds(args.train_seeds, rank, world)
    pairs, dns_ms = make_pairs(seeds, args, device=local)
    net = Net(seed=args.net_seed, device=local)
    tau_rms, hist = train_dp(net, pairs, args.iters, args.lr, group)
    t = torch.tensor([dns_ms], dtype=torch.float64, device="cuda")
    if group is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    if rank == 0:
        np.save(args.out, net.w.cpu().numpy())
        print(json.dumps({"ranks": world, "seeds": args.train_seeds, "pairs_per_rank": len(pairs),
                          "tau_rms": tau_rms, "loss_first": hist[0], "loss_last": hist[-1],
                          "data_gpu_ms_max_rank": float(t.item()), "weights": args.out}), flush=True)
    if group is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
