"""Learned JCG initial guess: parameters, training and evaluation drivers.

The network and its training run on the device (csrc/mpnn.cu, exposed
through adc_set_predictor / adc_predictor_train / adc_get_predictor); this
module holds the host side:

* the flat FP32 parameter layout, initialisation and the feature scales;
* `train`: trains on (state, solved ETAS) pairs that the plain FP64 solver
  produces on the surge mesh under seeded vortex tracks (central pressure
  920-980 hPa, Rmax 20-60 km, heading within 30 degrees of north), each
  track contributing a window of consecutive time steps at its own phase of
  the storm;
* `evaluate`: runs held-out tracks with the plain guess and with the
  learned guess (ADC_LEARNED_START) side by side and reports JCG
  iterations per step, the fallback rate and max |d eta| against the plain
  FP64 run.

    python -m adcirc_b200.learned train --out adcirc_b200/data/mpnn_surge.npz
    python -m adcirc_b200.learned evaluate --weights adcirc_b200/data/mpnn_surge.npz
"""
from __future__ import annotations

import argparse
import copy
import json
import math
import pathlib
import time

import numpy as np

from . import _lib, model

NF, F, H, L = 9, 16, 64, 3
OFF_WIN = 0
OFF_LAYER = OFF_WIN + H * F
LAYER_SZ = 2 * H * H + H
OFF_WOUT = OFF_LAYER + L * LAYER_SZ
OFF_BOUT = OFF_WOUT + H
OFF_NORM = OFF_BOUT + 1
NPARAMS = OFF_NORM + 2 * NF + 1
FEATURES = ("eta^k", "ETAS_ref", "u", "v", "depth", "wet", "p - p_bg", "tau_x", "tau_y")
DEFAULT_WEIGHTS = pathlib.Path(__file__).resolve().parent / "data" / "mpnn_surge.npz"


def layer_views(p: np.ndarray):
    """Named views into a flat parameter vector."""
    v = {"W_in": p[OFF_WIN:OFF_WIN + H * F].reshape(H, F)}
    for l in range(L):
        o = OFF_LAYER + l * LAYER_SZ
        v[f"Ws{l}"] = p[o:o + H * H].reshape(H, H)
        v[f"Wn{l}"] = p[o + H * H:o + 2 * H * H].reshape(H, H)
        v[f"b{l}"] = p[o + 2 * H * H:o + LAYER_SZ]
    v["w_out"] = p[OFF_WOUT:OFF_WOUT + H]
    v["b_out"] = p[OFF_BOUT:OFF_BOUT + 1]
    v["mean"] = p[OFF_NORM:OFF_NORM + NF]
    v["std"] = p[OFF_NORM + NF:OFF_NORM + 2 * NF]
    v["s_out"] = p[OFF_NORM + 2 * NF:OFF_NORM + 2 * NF + 1]
    return v


def features(arrays: dict, prbckgrnd: float) -> np.ndarray:
    """The nine node features the device computes before each solve, from
    host arrays holding the state at that point (ETA1 = eta^k, ETAS = the
    reference guess)."""
    a = arrays
    return np.stack([a["eta1"], a["etas"], a["uu1"], a["vv1"], a["dp"],
                     a["nodecode"].astype(np.float64), a["pr2"] - prbckgrnd, a["wsx2"], a["wsy2"]],
                    axis=1)


def init_params(mean, std, s_out, seed: int = 0) -> np.ndarray:
    """He-initialised weights with a zero head, so the first guess equals
    the reference guess."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, np.float32)
    v = layer_views(p)
    v["W_in"][:, :NF + 1] = rng.normal(0.0, math.sqrt(2.0 / (NF + 1)), (H, NF + 1))
    for l in range(L):
        v[f"Ws{l}"][:] = rng.normal(0.0, math.sqrt(1.0 / H), (H, H))
        v[f"Wn{l}"][:] = rng.normal(0.0, math.sqrt(1.0 / H), (H, H))
    v["mean"][:] = mean
    v["std"][:] = np.where(np.asarray(std) > 0, std, 1.0)
    v["s_out"][:] = s_out
    return p


def track(rng, base_case, hours: float = 30.0) -> model.Vortex:
    """A seeded straight track: pc 920-980 hPa, Rmax 20-60 km, heading
    within 30 degrees of north, 5 m/s, from the surge case's start point."""
    lx = base_case.meta.get("lx", 1000e3)
    pc = rng.uniform(920.0, 980.0)
    rmax = rng.uniform(20.0, 60.0)
    heading = 90.0 + rng.uniform(-30.0, 30.0)
    v = model.straight_track(0.5 * lx + 1234.5, 300e3 + 678.9, heading, 5.0, pc, rmax, 1.3, hours=hours)
    v.meta = {"pc_hpa": pc, "rmax_km": rmax, "heading_deg": heading}
    return v


def use_mask(arrays) -> np.ndarray:
    """Nodes where the network predicts: wet and off the elevation boundary."""
    use = arrays["nodecode"] == 1
    use[arrays["nbd"] - 1] = False
    return use


def _stats_from(case, gpu, hours: float = 6.0, samples: int = 60):
    """Feature means/scales and the correction scale s_out from a plain run
    into the storm: s_out is the RMS, over `samples` consecutive steps and
    the wet interior nodes, of the change of the solved increment between
    steps (the correction the network predicts)."""
    start = int(round(hours * 3600 / case.params["dt"]))
    gpu.run(1, start)
    gpu.sync_to_host()
    a = case.arrays
    x = features(a, case.params["prbckgrnd_mh2o"])
    ss, cnt = 0.0, 0
    for k in range(samples):
        e0 = a["etas"].copy()
        use = use_mask(a)
        gpu.run(1 + start + k, 1)
        gpu.sync_to_host()
        ss += float(np.sum((a["etas"][use] - e0[use]) ** 2))
        cnt += int(use.sum())
    s_out = math.sqrt(ss / max(cnt, 1)) or 1e-6
    return x.mean(axis=0), x.std(axis=0), s_out


def train(out: pathlib.Path, n_tracks: int = 8, pairs: int = 20000, seed: int = 7,
          lr: float = 1e-3, raw=None, log=print) -> dict:
    """Trains on `pairs` (state, solution) pairs, pairs / n_tracks
    consecutive steps per track, track k's window starting at hour
    1 + 3 k of its storm."""
    from . import meshgen
    rng = np.random.default_rng(seed)
    raw = raw if raw is not None else meshgen.surge_mesh()
    base = model.surge_case(raw=copy.deepcopy(raw))
    per = pairs // n_tracks
    g0 = model.GpuModel(base.clone())
    mean, std, s_out = _stats_from(g0.case, g0)
    g0.close()
    params = init_params(mean, std, s_out, seed)
    hist = []
    t0 = time.time()
    for k in range(n_tracks):
        c = base.clone()
        c.vortex = track(rng, base)
        gpu = model.GpuModel(c)
        start = int(round((1 + 3 * k) * 3600 / c.params["dt"]))
        gpu.run(1, start)
        gpu.set_predictor(params)
        gpu.predictor_train(True, lr)
        losses = []
        done = 0
        while done < per:
            n = min(500, per - done)
            gpu.run(1 + start + done, n)
            done += n
            losses.append(gpu.predictor_stats()[0])
        params = gpu.get_predictor()
        rec = {"track": k, **c.vortex.meta, "start_hour": 1 + 3 * k, "steps": per,
               "loss_first": losses[0], "loss_last": losses[-1], "adam_steps": gpu.predictor_stats()[1]}
        hist.append(rec)
        log(json.dumps(rec))
        gpu.close()
    out = pathlib.Path(out)
    out.parent.mkdir(parents=True, exist_ok=True)
    np.savez(out, params=params, history=json.dumps(hist), seed=seed, pairs=pairs,
             n_tracks=n_tracks, lr=lr)
    return {"history": hist, "seconds": time.time() - t0}


def load(path=DEFAULT_WEIGHTS) -> np.ndarray:
    d = np.load(path)
    p = np.asarray(d["params"], np.float32)
    if p.size != NPARAMS:
        raise ValueError(f"{path}: {p.size} parameters, expected {NPARAMS}")
    return p


def evaluate(params: np.ndarray, n_tracks: int = 4, seed: int = 1234, hours: int = 3,
             start_hour: int = 0, raw=None, log=print) -> dict:
    """Held-out tracks: plain guess vs learned guess from the same state,
    `hours` simulated hours each."""
    from . import meshgen
    rng = np.random.default_rng(seed)
    raw = raw if raw is not None else meshgen.surge_mesh()
    base = model.surge_case(raw=copy.deepcopy(raw))
    spd = int(round(3600 / base.params["dt"]))
    out = []
    for k in range(n_tracks):
        vt = track(rng, base)
        cp, cl = base.clone(), base.clone()
        cp.vortex = vt
        cl.vortex = vt
        gp = model.GpuModel(cp)
        gl = model.GpuModel(cl, prec=_lib.ADC_LEARNED_START)
        gl.set_predictor(params)
        it = 1
        if start_hour:
            gp.run(1, start_hour * spd)
            gl.run(1, start_hour * spd)
            it += start_hour * spd
        u0, f0 = gl.warm_start_stats()
        rec = {"track": k, **vt.meta, "hours": []}
        for h in range(hours):
            ip, _ = gp.run(it, spd)
            msp = gp.last_run_ms()
            il, _ = gl.run(it, spd)
            msl = gl.last_run_ms()
            it += spd
            gp.sync_to_host()
            gl.sync_to_host()
            d = np.abs(cl.arrays["eta2"] - cp.arrays["eta2"])
            u, f = gl.warm_start_stats()
            rec["hours"].append({"hour": start_hour + h + 1,
                                 "iters_plain": float(np.mean(ip)), "iters_learned": float(np.mean(il)),
                                 "ms_plain": msp / spd, "ms_learned": msl / spd,
                                 "fallback_rate": (f - f0) / max(u - u0 + f - f0, 1),
                                 "max_deta_m": float(d.max()),
                                 "wetdry_mismatch": int((cl.arrays["nodecode"] != cp.arrays["nodecode"]).sum())})
            u0, f0 = u, f
        log(json.dumps(rec))
        out.append(rec)
        gp.close()
        gl.close()
    return {"tracks": out}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("--out", default=str(DEFAULT_WEIGHTS))
    ap.add_argument("--weights", default=str(DEFAULT_WEIGHTS))
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--tracks", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--hours", type=int, default=3)
    ap.add_argument("--start-hour", type=int, default=0)
    args = ap.parse_args()
    from . import build
    build.build()
    if args.cmd == "train":
        r = train(pathlib.Path(args.out), n_tracks=args.tracks, pairs=args.pairs, lr=args.lr)
        print(json.dumps({"seconds": r["seconds"]}))
    else:
        r = evaluate(load(args.weights), hours=args.hours, start_hour=args.start_hour)
        print(json.dumps(r))


if __name__ == "__main__":
    main()
