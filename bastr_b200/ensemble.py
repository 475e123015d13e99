"""Batched ensemble of independent realizations (the C ABI's ``bastr_ensemble_*``).

Each realization has its own grid size, initial field seed and forcing; ``BastrEnsemble``
advances all of them together, a batch of steps being one CUDA-graph launch on the GPU.
``ensemble_configs`` builds the standard 96-member ensemble (32 each at 256^2, 512^2, 1024^2,
seeds 0-95, band forcing with forcek in {3..8} and targetenergy in [0.05, 0.1], FP32), and
``partition_by_cost`` splits realizations over GPUs by their estimated cost N log N (the
realizations are independent: no data crosses GPUs).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np


def ensemble_configs(n_per_size: int = 32, sizes=(256, 512, 1024), precision: str = "fp32",
                     steps_seed: int = 12345, **common) -> list[dict]:
    """Parameters of the standard ensemble: n_per_size realizations per grid size, seeds 0..,
    forcemethod 2 with forcek drawn uniformly from {3..8} and targetenergy from [0.05, 0.1]
    (numpy PCG64 seeded with `steps_seed`)."""
    rng = np.random.default_rng(steps_seed)
    out = []
    seed = 0
    for n in sizes:
        for _ in range(n_per_size):
            cfg = dict(ia=n, ja=n, ka=0, reynolds=5000.0, deltat=1e-4, forcemethod=2,
                       forcek=int(rng.integers(3, 9)), target_energy=float(rng.uniform(0.05, 0.1)),
                       lprojectd=True, precision=precision, velgrad_every=1, seed=seed, k0=4.0)
            cfg.update(common)
            out.append(cfg)
            seed += 1
    return out


def realization_cost(cfg: dict) -> float:
    """Estimated cost of one step: N log2 N grid points."""
    n = cfg["ia"] * cfg["ja"] * max(cfg.get("ka", 0), 1)
    return n * math.log2(n)


def partition_by_cost(configs: list[dict], world: int) -> list[list[int]]:
    """Longest-processing-time-first split of the realizations over `world` GPUs: indices per
    rank, each rank's total cost as even as the greedy rule makes it; deterministic."""
    order = sorted(range(len(configs)), key=lambda i: (-realization_cost(configs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += realization_cost(configs[i])
    return [sorted(p) for p in parts]


_PARAM_KEYS = ("ref_tem", "reynolds", "deltat", "kmax", "timemethod", "forcemethod", "forcek",
               "target_energy", "lprojectd", "precision", "device", "velgrad_every")


class BastrEnsemble:
    """Realizations advanced together on one GPU.  `configs`: one dict per realization with
    ia, ja, ka and any BastrGPU keyword (extra keys such as seed are ignored)."""

    def __init__(self, configs: list[dict], device: int = 0):
        from . import BastrError, CParams, load_library, make_cparams
        self._BastrError = BastrError
        self.lib = load_library()
        self.n = len(configs)
        arr = (CParams * self.n)()
        self.shapes = []
        self.ndims = []
        for i, c in enumerate(configs):
            kw = {k: c[k] for k in _PARAM_KEYS if k in c}
            kw["device"] = device
            arr[i] = make_cparams(c["ia"], c["ja"], c.get("ka", 0), **kw)
            ka = c.get("ka", 0)
            self.shapes.append((c["ja"], c["ia"]) if ka == 0 else (ka, c["ja"], c["ia"]))
            self.ndims.append(2 if ka == 0 else 3)
        self.e = C.c_void_p()
        rc = self.lib.bastr_ensemble_create(arr, self.n, C.byref(self.e))
        if rc != 0:
            msg = self._err()
            self.close()
            raise BastrError(rc, msg)

    def _err(self) -> str:
        buf = C.create_string_buffer(1024)
        if self.e:
            self.lib.bastr_ensemble_last_error(self.e, buf, 1024)
        return buf.value.decode(errors="replace")

    def _check(self, rc: int):
        if rc != 0:
            raise self._BastrError(rc, self._err())

    def close(self):
        if getattr(self, "e", None) and self.e.value:
            self.lib.bastr_ensemble_destroy(self.e)
            self.e = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_state(self, i: int, u):
        from . import _dptr
        arrs = [np.ascontiguousarray(c, dtype=np.float64).reshape(self.shapes[i]) for c in u]
        u3 = arrs[2] if self.ndims[i] == 3 else arrs[0]
        self._check(self.lib.bastr_ensemble_set_state(self.e, i, _dptr(arrs[0]), _dptr(arrs[1]), _dptr(u3)))

    def get_state(self, i: int):
        from . import _dptr
        out = [np.empty(self.shapes[i], dtype=np.float64) for _ in range(self.ndims[i])]
        u3 = out[2] if self.ndims[i] == 3 else out[0]
        self._check(self.lib.bastr_ensemble_get_state(self.e, i, _dptr(out[0]), _dptr(out[1]), _dptr(u3)))
        return out

    def step(self, nsteps: int):
        """Advances every realization by nsteps (at most 256 per call); returns the records,
        one list per realization."""
        from . import BastrGPU, CStepOut
        out = (CStepOut * max(self.n * nsteps, 1))()
        rc = self.lib.bastr_ensemble_step(self.e, nsteps, out)
        recs = [[BastrGPU._rec(out[i * nsteps + j]) for j in range(nsteps)] for i in range(self.n)]
        if rc != 0:
            raise self._BastrError(rc, self._err())
        return recs

    def run(self, nsteps: int, batch: int = 10) -> float:
        """Advances every realization by nsteps (a multiple of batch) as replays of the batch graph;
        returns the device time in ms (events on the ensemble's stream around all replays)."""
        ms = C.c_double()
        self._check(self.lib.bastr_ensemble_run(self.e, nsteps, batch, C.byref(ms)))
        return ms.value

    def subgrid(self, i: int, r: int):
        """(ub, tau) of realization i's current state as float32 CUDA tensors (bastr_ensemble_subgrid):
        the batched solver's closure training data."""
        import torch
        shape = [self.ndims[i]] + [n // r for n in self.shapes[i]]
        ub = torch.empty(shape, dtype=torch.float32, device="cuda")
        tau = torch.empty_like(ub)
        self._check(self.lib.bastr_ensemble_subgrid(self.e, i, r, C.c_void_p(ub.data_ptr()),
                                                    C.c_void_p(tau.data_ptr())))
        return ub, tau

    def set_plan(self, share_log2: int, i: int = -1):
        self._check(self.lib.bastr_ensemble_set_plan(self.e, i, share_log2))

    def plans(self) -> list[int]:
        a = (C.c_int32 * self.n)()
        self._check(self.lib.bastr_ensemble_get_plan(self.e, a))
        return list(a)

    def tune(self, nsteps: int = 4, reps: int = 2, max_share_log2: int = 3) -> float:
        """Autotunes the plans (state restored); returns the tuned time per step in ms."""
        ms = C.c_double()
        self._check(self.lib.bastr_ensemble_tune(self.e, nsteps, reps, max_share_log2, C.byref(ms)))
        return ms.value
