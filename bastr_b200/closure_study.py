"""A-posteriori study of the learned closure: filtered DNS against a coarse solve with and
without the closure, per spectrum shell, with the GPU time of each run.

    python -m bastr_b200.closure_study [--fine 256] [--ratio 4] [--train-seeds 0 1] [--test-seed 7]
                                       [--spinup 400] [--every 100] [--snapshots 4] [--steps 400]
                                       [--iters 2000] [--out FILE]

1. Training data from the batched solver: one fine realization per training seed (linear forcing,
   FP32 form) in one ensemble, advanced by CUDA-graph replays; after `--spinup` steps, every
   `--every` steps each realization's filtered field and subgrid term are formed on the device
   (bastr_ensemble_subgrid): pairs (ub, tau = filter(u.grad u) - ub.grad ub).
2. The network is trained on those pairs (tau scaled by its RMS) by the library's kernels.
3. Test: a fine run from the held-out seed; at the end of its spin-up its filtered field starts
   two coarse runs (same dt), one plain and one with the closure sub-step after every step.
   After `--steps` more steps the coarse runs' shell spectra are compared with the spectra of
   the filtered fine field (all three on the coarse grid, through the coarse solver's own
   spectra).  The held-out filtered state also gives the a-priori error of the network's tau.
   Prints one JSON object.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def _device_ms(stream, fn):
    """Device time in ms of the work fn() enqueues on `stream` (CUDA events on that stream)."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream.synchronize()
    e0.record(stream)
    out = fn()
    e1.record(stream)
    stream.synchronize()
    return out, e0.elapsed_time(e1)


def _advance(s, n):
    """n steps on a handle without reading records back (chunks of at most 256)."""
    while n > 0:
        c = min(n, 256)
        s.step_async(c)
        n -= c


def run(args) -> dict:
    import torch
    from . import BastrEnsemble, BastrGPU, seeded_field
    from .closure import Net

    nf, r = args.fine, args.ratio
    nc = nf // r
    phys = dict(reynolds=args.reynolds, deltat=args.dt, forcemethod=1, target_energy=args.target)
    batch = args.batch
    if args.spinup % batch or args.every % batch:
        raise ValueError("spinup and every must be multiples of batch")
    stream = torch.cuda.Stream()

    def fine_solver():
        s = BastrGPU(nf, nf, nf, precision="fp32", velgrad_every=0, kmax=nf // 3, **phys)
        s.set_stream(stream.cuda_stream)
        return s

    # 1. training pairs, made by the batched solver: one fine realization per training seed, advanced
    #    together by CUDA-graph replays; at every snapshot each realization's filtered field and
    #    subgrid term are formed on the device (bastr_ensemble_subgrid)
    #    (in ensembles of at most --group realizations, one after another, to bound device memory)
    pairs = []
    dns_ms = 0.0
    group = args.group if args.group > 0 else len(args.train_seeds)
    for g0 in range(0, len(args.train_seeds), group):
        seeds = args.train_seeds[g0:g0 + group]
        cfgs = [dict(ia=nf, ja=nf, ka=nf, precision="fp32", velgrad_every=0, kmax=nf // 3, seed=sd, **phys)
                for sd in seeds]
        with BastrEnsemble(cfgs) as ens:
            for i, sd in enumerate(seeds):
                ens.set_state(i, seeded_field(nf, nf, nf, k0=args.k0, seed=sd))
            dns_ms += ens.run(args.spinup, batch)
            for _ in range(args.snapshots):
                dns_ms += ens.run(args.every, batch)
                pairs += [ens.subgrid(i, r) for i in range(len(cfgs))]
    tau_rms = float(torch.sqrt(torch.mean(torch.stack([t for _, t in pairs]) ** 2)).item())
    train = [(ub.contiguous(), (t / tau_rms).contiguous()) for ub, t in pairs]

    # 2. training, by the library's forward / backward / Adam kernels
    net = Net(seed=args.net_seed)
    cur = torch.cuda.current_stream()
    hist, t_train = _device_ms(cur, lambda: net.train(train, iters=args.iters, lr=args.lr))

    # 3. test: the held-out fine run (the reference solution), and two coarse runs from its
    # filtered field
    def coarse_spectrum(fields):
        with BastrGPU(nc, nc, nc, **phys) as c:
            c.set_state(fields)
            _, es, ed, _ = c.spectra()
        return es + ed

    with fine_solver() as s:
        s.set_state(seeded_field(nf, nf, nf, k0=args.k0, seed=args.test_seed))
        _advance(s, args.spinup)
        ub0 = [c for c in s.subgrid(r)[0].cpu().numpy().astype(np.float64)]
        _, t_fine = _device_ms(stream, lambda: _advance(s, args.steps))
        ub1, tau1 = (x.cpu().numpy() for x in s.subgrid(r))   # held-out pair for the a-priori error
    e_dns = coarse_spectrum([c.astype(np.float64) for c in ub1])

    def coarse_run(closure: bool):
        with BastrGPU(nc, nc, nc, precision="fp32", velgrad_every=0, **phys) as c:
            c.set_stream(stream.cuda_stream)
            c.set_state(ub0)

            def go():   # no host round trip per step: records are not read back
                for i in range(args.steps):
                    c.step_async(1)
                    if closure and (i + 1) % args.closure_every == 0:
                        # one split sub-step covering the last closure_every steps
                        c.closure_apply(net, tau_rms, args.dt * args.closure_every)
            _, t = _device_ms(stream, go)
            return coarse_spectrum(c.get_state()), t

    e_plain, t_plain = coarse_run(False)
    e_clos, t_clos = coarse_run(True)
    kc = len(e_dns) - 1

    def err(e):
        rel = np.abs(e[1:kc] - e_dns[1:kc]) / e_dns[1:kc]
        return {"max_rel": float(rel.max()), "mean_rel": float(rel.mean()),
                "shells_within_5pct": int((rel <= 0.05).sum()), "shells": int(rel.size)}

    pred = net.forward(torch.tensor(ub1, device="cuda"), scale=tau_rms).cpu().numpy()
    apriori = {"mse_closure": float(np.mean((pred - tau1) ** 2)), "mse_no_closure": float(np.mean(tau1 ** 2))}
    return {
        "fine": nf, "coarse": nc, "filter_width_cells": r, "reynolds": args.reynolds, "dt": args.dt,
        "train_seeds": args.train_seeds, "test_seed": args.test_seed, "pairs": len(pairs),
        "spinup_steps": args.spinup, "test_steps": args.steps, "iters": args.iters, "tau_rms": tau_rms,
        "closure_every": args.closure_every, "training_data": "batched solver (bastr_ensemble_run + bastr_ensemble_subgrid)",
        "loss_first": hist[0], "loss_last": hist[-1], "train_gpu_ms": t_train, "training_dns_gpu_ms": dns_ms,
        "fine_gpu_ms": t_fine, "coarse_plain_gpu_ms": t_plain, "coarse_closure_gpu_ms": t_clos,
        "speedup_closure_vs_fine": t_fine / t_clos,
        "E_dns": e_dns[1:kc].tolist(), "E_plain": e_plain[1:kc].tolist(), "E_closure": e_clos[1:kc].tolist(),
        "error_plain": err(e_plain), "error_closure": err(e_clos), "apriori_held_out": apriori,
        "timing": "device time: CUDA events on the stream the runs launch on",
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--fine", type=int, default=256)
    ap.add_argument("--ratio", type=int, default=4)
    ap.add_argument("--reynolds", type=float, default=40.0)
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--target", type=float, default=1.5)
    ap.add_argument("--k0", type=float, default=3.0)
    ap.add_argument("--train-seeds", type=int, nargs="+", default=[0, 1])
    ap.add_argument("--test-seed", type=int, default=7)
    ap.add_argument("--spinup", type=int, default=400)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--snapshots", type=int, default=4)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--iters", type=int, default=2000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--net-seed", type=int, default=0)
    ap.add_argument("--batch", type=int, default=10, help="steps per CUDA-graph replay of the training ensemble")
    ap.add_argument("--group", type=int, default=0,
                    help="training realizations per ensemble (0: all in one); groups run one after another")
    ap.add_argument("--closure-every", type=int, default=1,
                    help="apply the closure once every this many coarse steps (sub-step dt times it)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    res = run(args)
    line = json.dumps(res)
    print(line, flush=True)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
