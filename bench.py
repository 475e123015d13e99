#!/usr/bin/env python
"""Throughput of the B200 pseudo-spectral Burgers time step (steps/s and HBM roofline).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload: 2D forced Burgers 2048x2048 (band forcing forcek=5, target 0.075,
lproject=t, dt=1e-4, Re=5000) in the FP32 form (FP32 fields/transforms/product, FP64 state,
spectra, energy and forcing reductions), with the reference's per-step diagnostics (shell
spectra and velocity-gradient statistics every step).  The same line carries the FP64 form and
the 3D 256^3 (linear forcing) forms as ``variants``.

A step is one iteration of the reference's main loop (spectra, velgrad, RK3, forcing).  The
single-field solver does not shard: ``--gpus N`` runs N independent replicas (weak scaling)
and ``value`` is the sum of their steps/s, timed on the device as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/s & %HBM roofline, 2048² and 256³: FP32 vs FP64 on GPU at ≤1e-5 rel err"

WORKLOADS = {
    "2d2048": dict(ia=2048, ja=2048, ka=0, reynolds=5000.0, ref_tem=273.15, deltat=1e-4, forcemethod=2,
                   forcek=5, target_energy=0.075, lprojectd=True, kmax=1 << 30, k0=4.0,
                   desc="2D forced Burgers 2048x2048, forcemethod=2 (forcek=5, target 0.075), lproject=t, "
                        "Re=5000, dt=1e-4, seeded k^4 exp(-2(k/4)^2) field, spectra+velgrad every step"),
    "3d256": dict(ia=256, ja=256, ka=256, reynolds=5000.0, ref_tem=273.15, deltat=5e-4, forcemethod=1,
                  forcek=5, target_energy=1.5, lprojectd=False, kmax=85, k0=3.0,
                  desc="3D forced Burgers 256^3, forcemethod=1 (target 1.5), Re=5000, dt=5e-4, spectra to "
                       "kmax=85, seeded k^4 exp(-2(k/3)^2) field, spectra+velgrad every step"),
}
HEADLINE = ("2d2048", "fp32")
VARIANTS = [("2d2048", "fp64"), ("3d256", "fp32"), ("3d256", "fp64")]


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def survey_bytes(w, prec):
    """Algorithmic bytes per step of the minimal fused c2c-free schedule: 66 V (2D), 171 V (3D),
    V = N * (4 or 8) bytes."""
    n = w["ia"] * w["ja"] * max(w["ka"], 1)
    v = n * (4 if prec == "fp32" else 8)
    return (66 if w["ka"] == 0 else 171) * v


# -------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# -------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock and throttle-reason samples (every 100 ms) around the timed region.

    A reader thread time-stamps every line as it arrives, so the samples taken while the GPU was
    loaded (between ``load_begin`` and ``load_end``) can be told apart from the start-up ones.
    ``wait_ready`` blocks until the first sample arrived, so that the loaded window is sampled."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []            # (time, fields)
        self.t_load = [None, None]
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.lines.append((time.perf_counter(), f))

    def wait_ready(self, timeout=5.0):
        t0 = time.perf_counter()
        while self.proc and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.02)

    def loaded_samples(self):
        a, b = self.t_load
        if a is None:
            return 0
        b = b if b is not None else time.perf_counter()
        return sum(1 for t, _ in self.lines if a <= t <= b)

    def load_begin(self):
        self.t_load[0] = time.perf_counter()

    def load_end(self):
        self.t_load[1] = time.perf_counter()

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "samples": 0, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        a, b = self.t_load
        sm, mx, pw, reasons = [], [], [], set()
        for t, f in self.lines:
            if a is not None and b is not None and not (a <= t <= b):
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                pw.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, f[5:9]):
                if v.lower() in ("active", "1", "yes"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "samples": len(sm), "reasons": sorted(reasons),
                "window": "samples taken while the solver stepped, the timed steps inside the window"}


# -------------------------------------------------------------------------------------------
# our arm
# -------------------------------------------------------------------------------------------
def make_solver(wl, prec, device):
    from bastr_b200 import BastrGPU
    w = WORKLOADS[wl]
    return BastrGPU(w["ia"], w["ja"], w["ka"], ref_tem=w["ref_tem"], reynolds=w["reynolds"],
                    deltat=w["deltat"], kmax=w["kmax"], forcemethod=w["forcemethod"], forcek=w["forcek"],
                    target_energy=w["target_energy"], lprojectd=w["lprojectd"], precision=prec,
                    device=device, velgrad_every=1)


def initial_field(wl):
    from bastr_b200 import seeded_field
    w = WORKLOADS[wl]
    return seeded_field(w["ia"], w["ja"], w["ka"], k0=w["k0"], seed=0)


def run_steps(s, n):
    while n > 0:
        c = min(n, 256)
        s.step_async(c)
        n -= c


def device_time(s, stream, nsteps, dist_ctx=None):
    """CUDA-event time of exactly nsteps steps on the library's stream (max over ranks)."""
    import torch
    if dist_ctx:
        dist_ctx.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run_steps(s, nsteps)
    e1.record(stream)
    s.sync()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist_ctx:
        ms = dist_ctx.max(ms)
        dist_ctx.barrier()
    return ms


def keep_loaded(s, seconds, chunk=20):
    """Untimed steps for about `seconds` of wall time (keeps the GPU loaded around the timed
    region while the clock sampler runs)."""
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        run_steps(s, chunk)
        s.sync()


def measure(wl, prec, steps, warmup, device, dist_ctx=None, sampler=None):
    """W untimed warm-up steps, then exactly `steps` timed steps.  With a clock sampler the GPU is
    kept loaded by untimed steps for about 0.6 s before and after the timed region (the same steps
    as the warm-up), so that the samples under load cover it even when it is a few milliseconds."""
    import torch
    s = make_solver(wl, prec, device)
    u = initial_field(wl)
    s.set_state(u)
    stream = torch.cuda.Stream(device=device)
    s.set_stream(stream.cuda_stream)
    run_steps(s, warmup)
    s.sync()
    if sampler:
        sampler.start()
        sampler.wait_ready()
        sampler.load_begin()
        keep_loaded(s, 0.6)
        # the loaded window advances the run by thousands of steps: the timed steps start again
        # from the seeded field, after the same warm-up, so they measure the configured run
        s.set_state(u)
        s.set_counters(0, 0.0)
        run_steps(s, warmup)
    ms = device_time(s, stream, steps, dist_ctx)
    clocks = None
    if sampler:
        t0 = time.perf_counter()
        keep_loaded(s, 0.6)
        while sampler.loaded_samples() < 10 and time.perf_counter() - t0 < 3.0:
            keep_loaded(s, 0.1)
        sampler.load_end()
        clocks = sampler.stop()
        s.set_state(u)
        s.set_counters(0, 0.0)
        run_steps(s, warmup)
        s.sync()
    info = s.info()
    return s, u, stream, ms, clocks, info


def kernel_roofline(s, nsteps, peak, peak_kind, wl, prec):
    stats = s.profile(nsteps)
    total = sum(k["total_ms"] for k in stats)
    top = max(stats, key=lambda k: k["total_ms"])
    per_launch_ms = top["total_ms"] / top["launches"]
    achieved = top["bytes_per_launch"] / (per_launch_ms * 1e-3) / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as f:
            t = json.load(f).get(f"{top['name']}@{wl}:{prec}")
            traffic = None if t is None else float(t)
    except Exception:
        pass
    shares = sorted(({"kernel": k["name"], "launches_per_step": k["launches"] / nsteps,
                      "share": round(k["total_ms"] / total, 4),
                      "gbs": round(k["bytes_per_launch"] / (k["total_ms"] / k["launches"] * 1e-3) / 1e9, 1)}
                     for k in stats), key=lambda d: -d["share"])
    return {"kernel": top["name"], "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
            "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} hbm_gbs",
            "algorithmic_bytes_per_launch": top["bytes_per_launch"], "traffic": traffic,
            "traffic_source": ("profiles/dram_traffic.json: ncu dram__bytes_read.sum + dram__bytes_write.sum "
                               "per launch from a capture of this kernel, not measured in this run")
            if traffic is not None else None,
            "share_of_step": round(top["total_ms"] / total, 4)}, shares


def fp32_accuracy(device, steps={"2d2048": 100, "3d256": 20}):
    """The FP32 form's error against the FP64 form on the GPU, per result, at the measured sizes:
    both forms step the same seeded field; relative L2 of the velocity, of each per-step scalar
    sequence and of every spectrum shell (worst step).  Untimed."""
    import numpy as np
    out = {}

    def rel(a, b):
        a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
        nb = np.linalg.norm(b)
        return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))

    for wl, n in steps.items():
        runs = {}
        for prec in ("fp64", "fp32"):
            s = make_solver(wl, prec, device)
            s.set_state(initial_field(wl))
            recs, sh = s.step(n, shells=True)
            runs[prec] = (recs, sh, np.stack(s.get_state()))
            s.close()
        (r64, s64, u64), (r32, s32, u32) = runs["fp64"], runs["fp32"]
        e = {"steps": n, "velocity": rel(u32, u64)}
        for name in ("Esspe", "Edspe", "k2Edspe", "kMEdspe", "factor"):
            e[name] = rel([getattr(r, name) for r in r32], [getattr(r, name) for r in r64])
        if math.isfinite(r64[0].E):
            e["E"] = rel([r.E for r in r32], [r.E for r in r64])
        vg = ("umumtheta2", "umumijji", "u2theta", "dissp", "eta_min", "Tay", "ReTay", "Kol")
        for i, name in enumerate(vg):
            e[name] = rel([r.velgrad[i] for r in r32], [r.velgrad[i] for r in r64])
        e["Es_shells"] = max(rel(s32[i, 0], s64[i, 0]) for i in range(n))
        e["Ed_shells"] = max(rel(s32[i, 1], s64[i, 1]) for i in range(n))
        e = {k: (float(f"{v:.3g}") if isinstance(v, float) else v) for k, v in e.items()}
        e["max_except_eta_min"] = max(v for k, v in e.items() if k not in ("steps", "eta_min"))
        out[wl] = e
    return out


def ensemble_measure(device, steps=1000, batch=10, seq_steps=100, peak=None, tune=True):
    """The standard ensemble (96 realizations: 32 each at 256^2, 512^2, 1024^2, seeds 0-95, band
    forcing with forcek in {3..8}, target in [0.05, 0.1], FP32), advanced `steps` steps as replays of
    one CUDA graph per batch of `batch` steps, device-timed (events on the ensemble's stream around
    all replays, BastrEnsemble.run).  Beside it: the same realizations stepped one after another
    through their own handles (device-timed per realization over `seq_steps` steps), and the device
    time of the closure training data (filtered field and subgrid term, r = 4) of one 1024^2
    realization.  B_model of an ensemble step: the sum of the realizations' 66 V (2D)."""
    import torch
    from bastr_b200 import BastrEnsemble, BastrGPU, ensemble_configs, seeded_field
    cfgs = ensemble_configs()
    fields = [seeded_field(c["ia"], c["ja"], 0, k0=c["k0"], seed=c["seed"]) for c in cfgs]
    out = {"realizations": len(cfgs), "sizes": sorted({c["ia"] for c in cfgs}), "precision": "fp32",
           "steps": steps, "batch": batch}
    with BastrEnsemble(cfgs, device=device) as ens:
        for i, u in enumerate(fields):
            ens.set_state(i, u)
        if tune:
            out["tuned_ms_per_step"] = round(ens.tune(nsteps=4, reps=2, max_share_log2=3), 4)
            out["plans_log2_by_size"] = {str(n): sorted({p for c, p in zip(cfgs, ens.plans()) if c["ia"] == n})
                                         for n in out["sizes"]}
            for i, u in enumerate(fields):
                ens.set_state(i, u)
        ens.run(3 * batch, batch)        # capture of the batch graph + warm-up
        ms = ens.run(steps, batch)
        i1024 = next(i for i, c in enumerate(cfgs) if c["ia"] == 1024)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ens.subgrid(i1024, 4)            # allocates the work buffers
        torch.cuda.synchronize()
        e0.record()
        ens.subgrid(i1024, 4)
        e1.record()
        torch.cuda.synchronize()
        out["subgrid_ms_1024"] = round(e0.elapsed_time(e1), 3)
    t_step = ms / steps
    out["device_ms_per_step"] = round(t_step, 4)
    out["ensemble_steps_per_s"] = round(1e3 / t_step, 2)
    out["realization_steps_per_s"] = round(len(cfgs) * 1e3 / t_step, 1)
    b_model = sum(66 * c["ia"] * c["ja"] * 4 for c in cfgs)
    out["b_model_bytes_per_step"] = b_model
    if peak:
        out["survey_roofline_frac"] = round(b_model / (t_step * 1e-3) / (peak * 1e9), 4)
    # one realization after another, each through its own handle, device-timed
    t_seq = 0.0
    for c, u in zip(cfgs, fields):
        with BastrGPU(c["ia"], c["ja"], 0, deltat=c["deltat"], forcemethod=2, forcek=c["forcek"],
                      target_energy=c["target_energy"], lprojectd=True, precision="fp32", device=device) as s:
            s.set_state(u)
            stream = torch.cuda.Stream(device=device)
            s.set_stream(stream.cuda_stream)
            run_steps(s, 3)
            s.sync()
            t_seq += device_time(s, stream, seq_steps) / seq_steps
    out["sequential_ms_per_step"] = round(t_seq, 4)
    out["sequential_realization_steps_per_s"] = round(len(cfgs) * 1e3 / t_seq, 1)
    out["timing"] = "CUDA events on the launching streams (device time), inputs resident"
    return out


def e2e_measure(wl, prec, steps, device):
    """Through the C ABI with host buffers: upload the field from pinned memory, step with the
    per-step records (scalars + shell spectra) read back every step, download the field."""
    import numpy as np
    import torch
    s = make_solver(wl, prec, device)
    u = initial_field(wl)
    pinned = [torch.empty(c.shape, dtype=torch.float64, pin_memory=True) for c in u]
    for p, c in zip(pinned, u):
        p.numpy()[...] = c
    host = [p.numpy() for p in pinned]
    host_out = [torch.empty(c.shape, dtype=torch.float64, pin_memory=True).numpy() for c in u]
    s.set_state(host)
    s.step(3, shells=True)   # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.set_state(host)
    for _ in range(steps):
        s.step(1, shells=True)
    out = s.get_state(out=host_out)
    t1 = time.perf_counter()
    state_bytes = sum(c.nbytes for c in u)
    rec_bytes = 8 * 16 + 2 * (s.allkmax + 1) * 8
    s.close()
    del out
    return {"value": round(steps / (t1 - t0), 3), "unit": "steps/s",
            "h2d_bytes_per_step": int(state_bytes / steps),
            "d2h_bytes_per_step": int(rec_bytes + state_bytes / steps),
            "note": "per step: bastr_step(1) with its scalar record and shell spectra read back; "
                    "field uploaded from pinned memory once and downloaded into pinned memory once per "
                    "timed run"}


def oracle_for(wl):
    from oracle.bastr_oracle import Oracle, Params
    w = WORKLOADS[wl]
    p = Params(ia=w["ia"], ja=w["ja"], ka=w["ka"], ref_tem=w["ref_tem"], reynolds=w["reynolds"],
               maxstep=1 << 30, deltat=w["deltat"], kmax=w["kmax"], forcemethod=w["forcemethod"],
               forcek=w["forcek"], target_energy=w["target_energy"], lprojectd=w["lprojectd"])
    cores = os.cpu_count() or 1
    o = Oracle(p, initial_field(wl), workers=cores)
    o.initial_dealias()
    return o, cores


def cpu_baseline(wl, max_seconds=20.0):
    """The FP64 c2c CPU oracle on the host cores, on a bounded sample of the same workload."""
    o, cores = oracle_for(wl)
    t = time.perf_counter()
    o.step_once(True)   # warm-up (plans, page-in)
    first = time.perf_counter() - t
    n = max(1, min(20, int(max_seconds / max(first, 1e-3))))
    t = time.perf_counter()
    for _ in range(n):
        o.step_once(True)
    dt = time.perf_counter() - t
    return {"value": round(n / dt, 5), "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": f"{n} full steps of {wl} (FP64 complex-to-complex restatement, scipy.fft workers={cores}) "
                      f"after 1 warm-up step"}


def whole_job_value(steps, ms_max, n_gpus):
    """Steps/s of the whole job: every replica ran ``steps`` steps; ``ms_max`` is the slowest
    rank's device time, so the job's throughput is n_gpus * steps over that time."""
    return n_gpus * steps / (ms_max * 1e-3)


class DistCtx:
    """One process per GPU (torchrun env): barrier and max-over-ranks of the device times.
    ``backend="gloo"`` runs the same host logic on CPU processes."""

    def __init__(self, backend="nccl"):
        import datetime
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.torch = torch
        self.backend = backend
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.local = int(os.environ.get("LOCAL_RANK", 0))
        if backend == "nccl":
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", self.local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))

    def barrier(self):
        self.dist.barrier()

    def max(self, v):
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = self.torch.tensor([v], dtype=self.torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        self.dist.destroy_process_group()


def ours(args):
    import torch
    n_gpus = args.gpus
    dist_ctx = DistCtx() if n_gpus > 1 else None
    rank = dist_ctx.rank if dist_ctx else 0
    device = dist_ctx.local if dist_ctx else 0
    torch.cuda.set_device(device)
    peak, peak_kind = hbm_peak()
    wl, prec = args.workload, args.precision
    w = WORKLOADS[wl]
    sampler = ClockSampler(device) if rank == 0 else None
    s, u, stream, ms, clocks, info = measure(wl, prec, args.steps, args.warmup, device, dist_ctx, sampler)
    steps_per_s = args.steps / (ms * 1e-3)
    value = whole_job_value(args.steps, ms, n_gpus)
    roof, shares = kernel_roofline(s, min(args.steps, 20), peak, peak_kind, wl, prec)
    s.close()
    variants = []
    if not args.no_variants:
        for vwl, vprec in VARIANTS:
            # about the same device time as the headline per variant
            vs, _, vstream, vms0, _, vinfo = measure(vwl, vprec, 5, 3, device, dist_ctx, None)
            ksteps = max(10, int(args.steps * (ms / args.steps) / (vms0 / 5)))
            vms = device_time(vs, vstream, ksteps, dist_ctx)
            vroof, _ = kernel_roofline(vs, min(ksteps, 5), peak, peak_kind, vwl, vprec)
            vs.close()
            vsps = ksteps / (vms * 1e-3)
            variants.append({"workload": vwl, "precision": vprec, "steps": ksteps, "steps_per_s": round(vsps, 2),
                             "ms_per_step": round(vms / ksteps, 4),
                             "mpoint_steps_per_s": round(vsps * WORKLOADS[vwl]["ia"] * WORKLOADS[vwl]["ja"]
                                                         * max(WORKLOADS[vwl]["ka"], 1) / 1e6, 1),
                             "survey_roofline_frac": round(survey_bytes(WORKLOADS[vwl], vprec) / (vms / ksteps * 1e-3)
                                                           / (peak * 1e9), 4),
                             "dominant_kernel": vroof})
    e2e = e2e_measure(wl, prec, max(20, min(args.steps, 200)), device) if (rank == 0 and not args.no_e2e) else None
    # the same end-to-end measure in the FP64 form, the reference's own precision
    e2e64 = (e2e_measure(wl, "fp64", max(20, min(args.steps, 200)), device)
             if (rank == 0 and not args.no_e2e and prec != "fp64") else None)
    ens = (ensemble_measure(device, peak=peak) if (rank == 0 and n_gpus == 1 and not args.no_variants
                                                  and not args.no_ensemble) else None)
    base = cpu_baseline(wl) if (rank == 0 and n_gpus == 1 and not args.no_cpu) else None
    acc = fp32_accuracy(device) if (rank == 0 and n_gpus == 1 and not args.no_variants) else None
    if dist_ctx:
        dist_ctx.barrier()
        dist_ctx.close()
    if rank != 0:
        return
    npts = w["ia"] * w["ja"] * max(w["ka"], 1)
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "steps/s", "n_gpus": n_gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if prec == "fp32" else "f64",
        "data": "synthetic (seeded Gaussian field, numpy PCG64 seed 0)",
        "config": {"workload": w["desc"],
                   "precision": "fp32 fields/FFTs/product, fp64 state+reductions+RK" if prec == "fp32" else "fp64",
                   "grid": [w["ia"], w["ja"], w["ka"]],
                   "parallelism": "replicas" if n_gpus > 1 else "single GPU, whole field resident",
                   "l2": "no flush: per-step working set and traffic exceed the 126 MB L2"},
        "mpoint_steps_per_s": round(steps_per_s * npts / 1e6, 1),
        "survey_roofline_frac": round(survey_bytes(w, prec) / (ms / args.steps * 1e-3) / (peak * 1e9), 4),
        "roofline": roof, "kernel_shares": shares, "variants": variants, "ensemble": ens,
        "cpu_baseline": base, "e2e": e2e, "e2e_fp64": e2e64,
        "fp32_vs_fp64_rel_l2": acc,
        "gpu_launches": int(info["launches_per_step"] * args.steps),
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def reference(args, budget_s=150.0):
    """The reference arm: the FP64 c2c CPU restatement of the reference's path (the Fortran
    reference cannot be built: no Fortran compiler, MPI, FFTW or HDF5), all host cores, on the
    headline workload.  Each step is one full main-loop step.  Exactly `--warmup` untimed and
    `--steps` timed steps run when they fit the time budget; otherwise fewer, and the line reports
    the counts that actually ran."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    wl, _ = HEADLINE
    o, cores = oracle_for(wl)
    t = time.perf_counter()
    o.step_once(True)                       # the first warm-up step (plans, page-in)
    first = time.perf_counter() - t
    fit = max(2, int(budget_s / max(first, 1e-3)))
    warmup = max(1, min(args.warmup, fit // 5))
    steps = max(1, min(args.steps, fit - warmup))
    for _ in range(warmup - 1):
        o.step_once(True)
    t = time.perf_counter()
    for _ in range(steps):
        o.step_once(True)
    dt = time.perf_counter() - t
    value = round(steps / dt, 5)
    base = {"value": value, "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": f"{steps} full steps of {wl} after {warmup} warm-up steps (FP64 complex-to-complex "
                      f"restatement, scipy.fft workers={cores})"}
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": "steps/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": warmup,
            "ms_per_step": round(1000.0 / base["value"], 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Gaussian field, numpy PCG64 seed 0)",
            "config": {"workload": WORKLOADS[wl]["desc"],
                       "implementation": "CPU restatement of the reference's FP64 FFTW c2c path (the Fortran "
                                         "reference cannot be built here: no Fortran compiler, MPI, FFTW or HDF5)"},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=HEADLINE[0],
                    help="headline workload (default: the 2048^2 band-forced case)")
    ap.add_argument("--precision", choices=["fp32", "fp64"], default=HEADLINE[1])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
