"""Shared helpers of the parity tests: run the oracle and the CUDA library on the same seeded
field and compare velocity, per-step scalars and every spectrum shell."""
from __future__ import annotations

import math

import numpy as np

from bastr_b200.initfield import seeded_field
from oracle.bastr_oracle import Oracle, Params


def make_params(ia, ja, ka=0, **kw) -> Params:
    return Params(ia=ia, ja=ja, ka=ka, **kw)


def run_oracle(p: Params, u, nsteps: int, velgrad: bool = True):
    o = Oracle(p, u)
    o.initial_dealias()
    recs, shells = [], []
    for _ in range(nsteps):
        rec, sp = o.step_once(velgrad)
        recs.append(rec)
        shells.append(np.stack([sp["Es"], sp["Ed"]]))
    return recs, np.array(shells), o.u


def run_gpu(p: Params, u, nsteps: int, precision: str = "fp64", velgrad: bool = True):
    from bastr_b200 import BastrGPU
    with BastrGPU(p.ia, p.ja, p.ka, ref_tem=p.ref_tem, reynolds=p.reynolds, deltat=p.deltat,
                  kmax=p.kmax, timemethod=p.timemethod, forcemethod=p.forcemethod, forcek=p.forcek,
                  target_energy=p.target_energy, lprojectd=p.lprojectd, precision=precision,
                  velgrad_every=1 if velgrad else 0) as s:
        s.set_state(u)
        recs, shells = s.step(nsteps, shells=True)
        uf = s.get_state()
    return recs, shells, uf


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def compare(ref, gpu, velgrad: bool = True):
    """Returns a dict of relative errors: velocity, each scalar sequence, shells (worst step)."""
    rrec, rsh, ru = ref
    grec, gsh, gu = gpu
    err = {"velocity": rel_l2(np.stack(gu), np.stack(ru))}
    for name in ("Esspe", "Edspe", "k2Edspe", "kMEdspe"):
        err[name] = rel_l2([getattr(r, name) for r in grec], [getattr(r, name) for r in rrec])
    if velgrad:
        names = ("umumtheta2", "umumijji", "u2theta", "dissp", "eta_min", "Tay", "ReTay", "Kol")
        for i, name in enumerate(names):
            err[name] = rel_l2([r.velgrad[i] for r in grec], [r.velgrad[i] for r in rrec])
    if rrec and rrec[0].forcing is not None:
        err["factor"] = rel_l2([r.factor for r in grec], [r.forcing[0] for r in rrec])
        if len(rrec[0].forcing) > 1:
            err["E"] = rel_l2([r.E for r in grec], [r.forcing[1] for r in rrec])
        if len(rrec[0].forcing) > 3:   # random-phase forcing also logs energy and Fen
            err["energy"] = rel_l2([r.energy for r in grec], [r.forcing[2] for r in rrec])
            err["Fen"] = rel_l2([r.Fen for r in grec], [r.forcing[3] for r in rrec])
    # every spectrum shell: relative L2 over the shell vector, worst over steps
    am = rsh.shape[-1]
    es = max(rel_l2(gsh[i, 0, :am], rsh[i, 0]) for i in range(len(rsh)))
    ed = max(rel_l2(gsh[i, 1, :am], rsh[i, 1]) for i in range(len(rsh)))
    err["Es_shells"] = es
    err["Ed_shells"] = ed
    for r in grec:
        assert math.isfinite(r.Esspe)
    return err


def compare_gpu_runs(ref, other, velgrad: bool = True):
    """Relative errors of one GPU run (`other`) against another (`ref`, e.g. the FP64 form):
    velocity, each per-step scalar, forcing factor and E, every spectrum shell (worst step)."""
    rrec, rsh, ru = ref
    grec, gsh, gu = other
    err = {"velocity": rel_l2(np.stack(gu), np.stack(ru))}
    names = ["Esspe", "Edspe", "k2Edspe", "kMEdspe", "factor"]
    if math.isfinite(rrec[0].E):   # forcing methods that log E (NaN in the record otherwise)
        names.append("E")
    for name in names:
        err[name] = rel_l2([getattr(r, name) for r in grec], [getattr(r, name) for r in rrec])
    if velgrad:
        vg = ("umumtheta2", "umumijji", "u2theta", "dissp", "eta_min", "Tay", "ReTay", "Kol")
        for i, name in enumerate(vg):
            err[name] = rel_l2([r.velgrad[i] for r in grec], [r.velgrad[i] for r in rrec])
    err["Es_shells"] = max(rel_l2(gsh[i, 0], rsh[i, 0]) for i in range(len(rsh)))
    err["Ed_shells"] = max(rel_l2(gsh[i, 1], rsh[i, 1]) for i in range(len(rsh)))
    for r in grec:
        assert math.isfinite(r.Esspe)
    return err


def field(ia, ja, ka=0, k0=4.0, seed=0):
    return seeded_field(ia, ja, ka, k0=k0, seed=seed)
