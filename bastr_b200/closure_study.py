"""A-posteriori study of the learned closure: filtered DNS against a coarse solve with and
without the closure, per spectrum shell, with the GPU time of each run.

    python -m bastr_b200.closure_study [--fine 256] [--ratio 4] [--train-seeds 0 1] [--test-seed 7]
                                       [--spinup 400] [--every 100] [--snapshots 4] [--steps 400]
                                       [--iters 2000] [--out FILE]

1. Training data: fine runs (linear forcing, FP32 form) from seeded fields; after `--spinup`
   steps, every `--every` steps the velocity and its advective term are box-filtered onto the
   coarse grid: pairs (ub, tau = filter(u.grad u) - ub.grad ub).
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
import time

import numpy as np


def _sync_time(fn):
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = fn()
    torch.cuda.synchronize()
    return out, time.perf_counter() - t0


def run(args) -> dict:
    import torch
    from . import BastrGPU, seeded_field
    from .closure import Net, box_filter, filtered_pair

    nf, r = args.fine, args.ratio
    nc = nf // r
    phys = dict(reynolds=args.reynolds, deltat=args.dt, forcemethod=1, target_energy=args.target)

    def fine_solver():
        return BastrGPU(nf, nf, nf, precision="fp32", velgrad_every=0, kmax=nf // 3, **phys)

    def dev(a):
        return torch.tensor(np.ascontiguousarray(a, np.float32), device="cuda")

    # 1. training pairs
    pairs = []
    for seed in args.train_seeds:
        with fine_solver() as s:
            s.set_state(seeded_field(nf, nf, nf, k0=args.k0, seed=seed))
            s.step(args.spinup)
            for _ in range(args.snapshots):
                s.step(args.every)
                pairs.append(filtered_pair(s, s.get_state(), r))
    tau_rms = float(np.sqrt(np.mean(np.stack([t for _, t in pairs]) ** 2)))
    train = [(dev(ub), dev(t / tau_rms)) for ub, t in pairs]

    # 2. training
    net = Net(seed=args.net_seed)
    hist, t_train = _sync_time(lambda: net.train(train, iters=args.iters, lr=args.lr))

    # 3. test
    def coarse_spectrum(fields):
        with BastrGPU(nc, nc, nc, **phys) as c:
            c.set_state(fields)
            _, es, ed, _ = c.spectra()
        return es + ed

    with fine_solver() as s:
        s.set_state(seeded_field(nf, nf, nf, k0=args.k0, seed=args.test_seed))
        s.step(args.spinup)
        ub0 = [box_filter(c, r) for c in s.get_state()]
        _, t_fine = _sync_time(lambda: s.step(args.steps))
        u1 = s.get_state()
        ub1, tau1 = filtered_pair(s, u1, r)   # held-out pair for the a-priori error
    e_dns = coarse_spectrum([box_filter(c, r) for c in u1])

    def coarse_run(closure: bool):
        with BastrGPU(nc, nc, nc, precision="fp32", velgrad_every=0, **phys) as c:
            c.set_state(ub0)

            def go():   # no host round trip per step: records are not read back
                for i in range(args.steps):
                    c.step_async(1)
                    if closure and (i + 1) % args.closure_every == 0:
                        # one split sub-step covering the last closure_every steps
                        c.closure_apply(net, tau_rms, args.dt * args.closure_every)
                c.sync()
            _, t = _sync_time(go)
            return coarse_spectrum(c.get_state()), t

    e_plain, t_plain = coarse_run(False)
    e_clos, t_clos = coarse_run(True)
    kc = len(e_dns) - 1

    def err(e):
        rel = np.abs(e[1:kc] - e_dns[1:kc]) / e_dns[1:kc]
        return {"max_rel": float(rel.max()), "mean_rel": float(rel.mean()),
                "shells_within_5pct": int((rel <= 0.05).sum()), "shells": int(rel.size)}

    pred = net.forward(dev(ub1), scale=tau_rms).cpu().numpy()
    apriori = {"mse_closure": float(np.mean((pred - tau1) ** 2)), "mse_no_closure": float(np.mean(tau1 ** 2))}
    return {
        "fine": nf, "coarse": nc, "filter_width_cells": r, "reynolds": args.reynolds, "dt": args.dt,
        "train_seeds": args.train_seeds, "test_seed": args.test_seed, "pairs": len(pairs),
        "spinup_steps": args.spinup, "test_steps": args.steps, "iters": args.iters, "tau_rms": tau_rms,
        "closure_every": args.closure_every,
        "loss_first": hist[0], "loss_last": hist[-1], "train_gpu_s": t_train,
        "fine_gpu_s": t_fine, "coarse_plain_gpu_s": t_plain, "coarse_closure_gpu_s": t_clos,
        "speedup_closure_vs_fine": t_fine / t_clos,
        "E_dns": e_dns[1:kc].tolist(), "E_plain": e_plain[1:kc].tolist(), "E_closure": e_clos[1:kc].tolist(),
        "error_plain": err(e_plain), "error_closure": err(e_clos), "apriori_held_out": apriori,
        "timing": "host wall time with device synchronisation around each run; coarse runs launch asynchronously",
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
