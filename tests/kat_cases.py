"""Cases for the known-answer tests (volume conservation, inflow mass
balance, mirror symmetry) shared by the oracle and GPU test files.

Each holds for the discrete GWCE itself, not only for the continuum
equations, so both implementations must meet it to solver tolerance:

* a closed, fully wet basin (no open boundary, no flux): every spatial term
  of the GWCE is in divergence form and the land boundary integral is zero,
  so summing the discrete equations (the basis functions sum to one) leaves
  V^{k+1} - 2V^k + V^{k-1} + tau0*dt/2*(V^{k+1} - V^{k-1}) = 0 for the
  volume V = sum_e A_e * mean(eta over e) (gwce.F:427-743, 1000-1617);
* the same basin with a steady specified inflow (IBTYPE 2, gwce.F:
  1737-1834): once the flux ramp is complete each step adds Q*dt;
* a channel triangulated mirror-symmetrically about its centreline,
  forced uniformly along the open boundary, without Coriolis: eta and u
  are even and v is odd under the mirror;
* the quarter-annular harbour of Lynch and Gray (depth ~ r^2, linear
  friction, M2 on the outer arc), whose periodic linear tide has a closed
  form (model.quarter_annulus_solution): the discrete solution matches it
  to discretisation error, which falls with refinement.
"""
from __future__ import annotations

import math

import numpy as np

NX, NY = 61, 21
LX, LY = 30e3, 10e3


def _nid(i, j):
    return i * NY + j


def basin_volume(case) -> float:
    a = case.arrays
    nm = a["nm"] - 1
    e = a["eta2"]
    return float(np.sum(0.5 * a["areas"] * (e[nm[:, 0]] + e[nm[:, 1]] + e[nm[:, 2]]) / 3.0))


def closed_basin(prep=None):
    """Closed basin 30 x 10 km, 20 -> 10 m deep, an initial 0.2 m hump."""
    from adcirc_b200 import meshgen, model
    raw = meshgen.channel_mesh(nx=NX, ny=NY, lx=LX, ly=LY, depth0=20.0, depth1=10.0)
    land = list(raw.land_segments[0][1]) + list(raw.open_nodes[1:])
    raw.land_segments = [(0, np.asarray(land, np.int64))]
    raw.open_nodes = np.array([], np.int64)
    eta0 = 0.2 * np.exp(-((raw.x - 10e3) ** 2 + (raw.y - 4e3) ** 2) / 3e3 ** 2)
    params = model.default_params(5.0, nolifa=1)
    return model.build_case(raw, params, model.Schedule(dt=5.0, nramp=0), [], eta0=eta0,
                            prep=prep)


RIVER_Q = 0.5            # m^2/s per unit width on the east end
RIVER_WIDTH = LY


def river_basin(prep=None):
    """The closed basin with a steady inflow through its east end."""
    from adcirc_b200 import meshgen, model
    raw = meshgen.channel_mesh(nx=NX, ny=NY, lx=LX, ly=LY, depth0=10.0, depth1=5.0)
    south = np.array([_nid(i, 0) for i in range(NX)])
    east = np.array([_nid(NX - 1, j) for j in range(NY)])
    north = np.array([_nid(i, NY - 1) for i in range(NX - 1, -1, -1)])
    west = np.array([_nid(0, j) for j in range(NY - 1, -1, -1)])
    raw.land_segments = [(0, south), (2, east), (0, np.concatenate([north, west[1:]]))]
    raw.open_nodes = np.array([], np.int64)
    params = model.default_params(5.0, nolifa=1)
    sched = model.Schedule(dt=5.0, dramp=0.5, dramp_extflux=0.02)
    case = model.build_case(raw, params, sched, [], prep=prep)
    lbc = case.arrays["lbcodei"]
    nv = lbc.size
    qnam = np.zeros((1, nv))
    qnam[0, (lbc == 2) | (lbc == 12) | (lbc == 22)] = RIVER_Q
    case.flux = model.Flux(np.zeros(1), np.zeros(1), np.ones(1), np.zeros(1), qnam,
                           np.zeros((1, nv)))
    return case


def inflow_volume(case, it0: int, it1: int) -> float:
    """Specified inflow volume of steps it0..it1-1 (ramped, dt each)."""
    s = case.schedule
    return sum(RIVER_Q * RIVER_WIDTH * s.step(k).rampextflux * s.dt for k in range(it0, it1))


def mirror_channel(prep=None):
    """Channel whose lower half has diagonals SW-NE and upper half NW-SE, so
    the triangulation is its own mirror image about y = LY/2; M2 tide on
    x = 0 uniform in y; CORI = 0."""
    from adcirc_b200 import meshgen, model
    raw = meshgen.channel_mesh(nx=NX, ny=NY, lx=LX, ly=LY, depth0=20.0, depth1=5.0)
    tris = []
    for i in range(NX - 1):
        for j in range(NY - 1):
            a, b, c, d = _nid(i, j), _nid(i + 1, j), _nid(i + 1, j + 1), _nid(i, j + 1)
            tris += [(a, b, c), (a, c, d)] if j < (NY - 1) // 2 else [(a, b, d), (b, c, d)]
    raw.nm = np.asarray(tris, np.int64)
    neta = raw.open_nodes.size
    tides = [(2.0 * math.pi / 44712.0, 0.0, 1.0, np.full(neta, 0.5), np.zeros(neta))]
    params = model.default_params(5.0)
    return model.build_case(raw, params, model.Schedule(dt=5.0, dramp=0.05), tides, cori=0.0,
                            prep=prep)


def mirror_index():
    k = np.arange(NX * NY)
    return (k // NY) * NY + (NY - 1 - k % NY)


def asymmetry(case) -> dict:
    a = case.arrays
    m = mirror_index()
    e, u, v = a["eta2"], a["uu2"], a["vv2"]
    return {"eta": float(np.abs(e - e[m]).max() / np.abs(e).max()),
            "u": float(np.abs(u - u[m]).max() / np.abs(u).max()),
            "v": float(np.abs(v + v[m]).max() / max(np.abs(v).max(), 1e-30))}


def harmonic_m2(step_fn, case, n_spin_days: float = 5.0, cycles: int = 2):
    """Runs `step_fn(it0, n)` (a model's run method) from cold start for
    n_spin_days, then samples ETA2 every step over `cycles` M2 periods and
    returns the least-squares M2 amplitude and phase (eta = A cos(w t -
    phase)) per node."""
    from adcirc_b200 import model
    w = 2.0 * math.pi / model.M2_PERIOD
    dt = case.params["dt"]
    n_spin = int(n_spin_days * 86400.0 / dt)
    per = int(round(model.M2_PERIOD / dt))
    step_fn(1, n_spin)
    it = n_spin + 1
    ts, etas = [], []
    for _ in range(cycles * per):
        step_fn(it, 1)
        ts.append(it * dt)
        etas.append(case.arrays["eta2"].copy())
        it += 1
    ts = np.asarray(ts)
    A = np.stack([np.cos(w * ts), np.sin(w * ts), np.ones_like(ts)], axis=1)
    coef, *_ = np.linalg.lstsq(A, np.asarray(etas), rcond=None)
    return np.hypot(coef[0], coef[1]), np.arctan2(coef[1], coef[0])


def annulus_errors(case, amp, phase):
    """Max relative amplitude error and max phase error [deg] against the
    closed-form quarter-annulus tide."""
    from adcirc_b200 import model
    r = np.hypot(case.arrays["x"], case.arrays["y"])
    ea, ep = model.quarter_annulus_solution(r, case.meta)
    dph = np.degrees(np.abs((phase - ep + np.pi) % (2.0 * np.pi) - np.pi))
    return float((np.abs(amp - ea) / ea).max()), float(dph.max())
