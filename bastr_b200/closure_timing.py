"""Device timing of the learned closure's kernels at 128^3 (CUDA events on the launching stream):
the tensor-core forward (bastr_net_forward), the loss and gradient (bastr_net_grad), a plain
128^3 FP32 step of the coarse solver and the closure sub-step on its state
(bastr_closure_apply).

    python -m bastr_b200.closure_timing [--n 128]
"""
from __future__ import annotations

import argparse
import json


def main():
    import torch

    from . import BastrGPU, seeded_field
    from .closure import Net

    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    args = ap.parse_args()
    n = args.n
    net = Net(seed=0)
    u = torch.randn(3, n, n, n, device="cuda")
    tau = torch.randn(3, n, n, n, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps, stream=None):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    out = {"points": n ** 3,
           "net_forward_ms": timed(lambda: net.forward(u), 20),
           "net_loss_grad_ms": timed(lambda: net.loss_grad(u, tau), 5)}
    with BastrGPU(n, n, n, reynolds=80.0, deltat=5e-4, forcemethod=1, target_energy=1.5, precision="fp32",
                  velgrad_every=0) as s:
        s.set_state(seeded_field(n, n, n, k0=3.0, seed=0))
        st = torch.cuda.Stream()
        s.set_stream(st.cuda_stream)

        def step():
            s.step_async(1)

        out["plain_step_ms"] = timed(step, 50, st)
        with torch.cuda.stream(st):
            out["closure_apply_ms"] = timed(lambda: s.closure_apply(net, 1.0, 5e-4), 20, st)
    out["timing"] = "CUDA events on the launching stream, after two untimed calls"
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
