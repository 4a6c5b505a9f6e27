"""Batched ensemble of storm-surge members (adc_ensemble_*).

Members: `n` surge meshes generated as the benchmark mesh (Poisson-disk,
graded to a seeded fractal coastline, shelf + random-field bathymetry)
with their own seeds and node counts drawn log-uniform from [50k, 400k];
each with M2 + K1 tides, wet/dry on and a perturbed Holland vortex
(central pressure 920-980 hPa, Rmax 20-60 km, forward speed 3-8 m/s,
heading within 30 degrees of north).

`Ensemble` binds every member as its own device context and steps them
together: one captured CUDA graph per time step holds all members' steps
on their own streams (adc_ensemble_run).  `autotune` chooses the JCG
row-block counts of the members (the persistent solvers are what limit
how much of the GPU the members can share) by timing a few candidate
layouts on the ensemble itself.
"""
from __future__ import annotations

import ctypes as C
import math
import multiprocessing as mp

import numpy as np

from . import _lib, model

# node count of the benchmark mesh at its grading (surge_mesh's bisection
# result) and the count's power-law response to the grading
_ALPHA600K, _N600K, _GAMMA = 0.03493, 599_676, 0.85


def _alpha_for(nodes: float) -> float:
    return _ALPHA600K * (_N600K / nodes) ** (1.0 / _GAMMA)


def _make_mesh(args):
    seed, nodes = args
    from . import meshgen
    raw = meshgen.surge_mesh(seed=seed, target_nodes=int(nodes), alpha=_alpha_for(nodes))
    raw.meta = {k: v for k, v in raw.meta.items() if k != "coast_fn"}   # picklable
    return raw


def member_specs(n: int = 48, seed: int = 5, nmin: float = 50e3, nmax: float = 400e3):
    """Per member: mesh seed, target node count (log-uniform), vortex."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        out.append({"mesh_seed": int(1000 + 17 * k + seed), "nodes": float(math.exp(rng.uniform(math.log(nmin),
                                                                                                 math.log(nmax)))),
                    "pc_hpa": float(rng.uniform(920.0, 980.0)), "rmax_km": float(rng.uniform(20.0, 60.0)),
                    "speed": float(rng.uniform(3.0, 8.0)), "heading": float(90.0 + rng.uniform(-30.0, 30.0))})
    return out


def build_members(specs, processes: int | None = None):
    """Member cases; meshes are generated in spawned worker processes."""
    args = [(s["mesh_seed"], s["nodes"]) for s in specs]
    procs = processes or max(1, min(len(args), mp.cpu_count()))
    if procs > 1:
        with mp.get_context("spawn").Pool(procs) as pool:
            raws = pool.map(_make_mesh, args, chunksize=1)
    else:
        raws = [_make_mesh(a) for a in args]
    cases = []
    for s, raw in zip(specs, raws):
        c = model.surge_case(raw=raw, vortex=False, nws=8)
        c.vortex = model.straight_track(0.5 * raw.meta["lx"] + 1234.5, 300e3 + 678.9, s["heading"],
                                        s["speed"], s["pc_hpa"], s["rmax_km"], 1.3, hours=30.0)
        cases.append(c)
    return cases


class Ensemble:
    """The members bound on the device and stepped as one graph per step.
    All members take the first member's step table (same DT, start time
    and ramps)."""

    def __init__(self, cases, prec: int = 0, predictor=None):
        self.lib = _lib.load()
        self.cases = cases
        self.models = [model.GpuModel(c, prec=prec) for c in cases]
        if predictor is not None:
            for m in self.models:
                m.set_predictor(predictor)
        self._arr = (C.c_void_p * len(self.models))(*[m.h.value for m in self.models])
        h = C.c_void_p()
        rc = self.lib.adc_ensemble_create(len(self.models), self._arr, C.byref(h))
        if rc != 0:
            raise model.AdcError(f"adc_ensemble_create: {rc}: {_lib.last_error()}")
        self.h = h
        self.it = 1
        self.schedule = cases[0].schedule

    @property
    def nodes(self) -> int:
        return int(sum(c.sizes["np"] for c in self.cases))

    def run(self, nsteps: int):
        steps = self.schedule.steps(self.it, nsteps)
        numitr = np.zeros((len(self.models), nsteps), np.int32)
        last = (_lib.AdcStepOut * len(self.models))()
        rc = self.lib.adc_ensemble_run(self.h, nsteps, steps, numitr.ctypes.data_as(_lib.ip_), last)
        if rc != 0:
            raise model.AdcError(f"adc_ensemble_run: status {rc}: {_lib.last_error()}")
        self.it += nsteps
        return numitr, float(self.lib.adc_ensemble_last_ms(self.h))

    def layouts(self):
        out = []
        for m in self.models:
            rb, res = C.c_int(0), C.c_int(0)
            self.lib.adc_jcg_layout(m.h, C.byref(rb), C.byref(res))
            out.append((rb.value, res.value))
        return out

    def set_row_blocks(self, blocks):
        for m, b in zip(self.models, blocks):
            rc = self.lib.adc_set_jcg_blocks(m.h, int(b))
            if rc != 0:
                raise model.AdcError(f"adc_set_jcg_blocks: {rc}: {_lib.last_error()}")

    def close(self):
        if self.h:
            self.lib.adc_ensemble_free(self.h)
            self.h = None
        for m in self.models:
            m.close()


def candidate_layouts(sizes, sm_count: int = 148):
    """JCG row blocks per member: each member's own default (0), and
    shares of one or two blocks per SM split in proportion to member size
    (every member at least one block)."""
    sizes = np.asarray(sizes, np.float64)
    cands = {"default": [0] * len(sizes)}
    for name, total in (("share_1x", sm_count), ("share_2x", 2 * sm_count - len(sizes))):
        b = np.maximum(1, np.floor(total * sizes / sizes.sum())).astype(int)
        cands[name] = b.tolist()
    return cands


def autotune(ens: Ensemble, steps: int = 30, log=print):
    """Times each candidate layout on `steps` ensemble steps (the ensemble
    advances meanwhile) and keeps the fastest."""
    sizes = [c.sizes["np"] for c in ens.cases]
    results = {}
    best, best_ms = None, float("inf")
    for name, blocks in candidate_layouts(sizes).items():
        ens.set_row_blocks(blocks)
        ens.run(3)                       # capture and warm up
        _, ms = ens.run(steps)
        results[name] = {"ms_per_step": ms / steps, "resident_members":
                         int(sum(r for _, r in ens.layouts()))}
        log(f"autotune {name}: {ms / steps:.3f} ms/step")
        if ms < best_ms:
            best, best_ms = name, ms
    ens.set_row_blocks(candidate_layouts(sizes)[best])
    return best, results


def sequential_step_ms(ens: Ensemble, steps: int = 20) -> float:
    """The same members stepped one after another (each member's own
    captured step graph, adc_run), for comparison: ms per ensemble step."""
    tot = 0.0
    for m in ens.models:
        m.run(ens.it, steps)
        tot += m.last_run_ms()
    ens.it += steps
    return tot / steps
