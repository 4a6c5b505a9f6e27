"""Throughput of the ADCIRC 2DDI time step on B200 (sim-days per wall-hour).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl adcgpu|reference]

A "step" is one ADCIRC time step (dt = 1 s) of the ~600k-node synthetic
surge mesh: friction and time-level shift, GWCE assembly, the JCG solve,
wetting/drying and the momentum update, all device resident.  The value is
simulated days per wall-clock hour over K timed steps after W warm-up
steps.  For N > 1 (torchrun) every rank runs an independent replica on its
own GPU (the path does not shard without a domain decomposition): value is
the aggregate over ranks, timed as the max over ranks.

--impl reference times the CPU restatement of the reference (the serial
FP64 oracle, the reference's own Fortran cannot be built on this image) on
a bounded sample of the same workload.
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
import pathlib

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "sim-days/wall-hour, 600k-node surge mesh: chosen vs plain FP64 GPU, Δη≤1mm"
UNIT = "sim-days/wall-hour"
HBM_FALLBACK_GBS = 6650.0


def forcing(case):
    """One-line description of the met forcing of a case."""
    v = getattr(case, "vortex", None)
    if v is None:
        return "no met forcing"
    f = v.fixes[0]
    return (f"Holland vortex NWS=8 (pc {f[3] / 100:.0f} hPa, Rmax {f[5]:.0f} km, "
            f"B 1.3, {np.hypot(f[6], f[7]):.0f} m/s straight track)")


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


def sim_days_per_hour(nsteps, dt, seconds):
    return (nsteps * dt / 86400.0) / (seconds / 3600.0)


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.samples = []
        self._p = None
        self._t = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self._p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._p = None
        return self

    def _read(self):
        for line in self._p.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self._p is not None:
            self._p.terminate()
            try:
                self._p.wait(timeout=5)
            except Exception:
                self._p.kill()
            if self._t:
                self._t.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if s[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def jcg_bytes(nnz_o: int, npn: int, iters: float, vbytes: int = 8) -> float:
    """Algorithmic HBM bytes of one JCG solve (persistent kernel), counted
    as a streaming implementation would move them.

    Per off-diagonal slot: the scaling pass, which also forms d0, reads the
    FP64 value + column and writes the scaled value (vbytes: 8, or 4 for the
    FP32 matrix copy); each later SpMV pass (dtwd0, one per iteration) reads
    value + 4 B column.
    Per row: prologue 64+44+24 B, 68 B per iteration (own record 32, u and
    u1 16, row length 4, writes 32+8 minus the neighbours' records counted
    once), epilogue 60 B.
    """
    slot = vbytes + 4.0
    return (nnz_o * (12.0 + vbytes + slot * (1.0 + iters)) +
            npn * (64.0 + 44.0 + 24.0 + 68.0 * iters + 60.0))


def profiled_traffic(kernel: str = "jcg_kernel<1, float>"):
    """DRAM bytes (read + write) of one launch of `kernel`, from the committed
    ncu summary profiles/surge_kernels_full.md, or None."""
    p = ROOT / "profiles" / "surge_kernels_full.md"
    if not p.exists():
        return None
    cols, vals = None, {}
    for line in p.read_text().splitlines():
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if line.startswith("| metric |"):
            cols = [c.strip("`") for c in cells[1:]]
        elif cols and line.startswith("| DRAM read") or cols and line.startswith("| DRAM write"):
            vals[cells[0]] = cells[1:]
    if not cols or kernel not in cols or len(vals) != 2:
        return None
    k = cols.index(kernel)
    try:
        return sum(float(v[k]) * 1e6 for v in vals.values())   # Mbyte -> bytes
    except (ValueError, IndexError):
        return None


def make_case(name: str):
    from adcirc_b200 import model
    if name == "surge":
        return model.surge_case()
    if name == "channel":
        return model.channel_case()
    raise ValueError(name)


def run_cpu_baseline(case, max_seconds: float = 20.0, min_steps: int = 2, it0: int = 1):
    """The oracle (serial FP64 restatement) on a bounded sample of steps."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    oracle.build()
    c = case.clone()
    om = oracle.OracleModel(c)
    t0 = time.perf_counter()
    n = 0
    its = []
    while True:
        its.append(om.step(it0 + n).numitr)
        n += 1
        el = time.perf_counter() - t0
        if (n >= min_steps and el >= max_seconds) or n >= 100000:
            break
    om.close()
    return n, el, its


def bench_reference(args, rank, world):
    if rank != 0:
        return
    case = make_case(args.case)
    dt = case.params["dt"]
    budget = min(90.0, max(10.0, 3.0 * (args.steps + args.warmup)))
    n, el, its = run_cpu_baseline(case, max_seconds=budget)
    v = sim_days_per_hour(n, dt, el)
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": n,
        "warmup": 0, "ms_per_step": 1000.0 * el / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": f"{args.case}: {case.sizes['np']} nodes, {case.sizes['ne']} elements, dt {dt} s, "
                               f"M2+K1 tides, {forcing(case)}, wet/dry on, plain FP64 JCG",
                   "parallelism": "serial (1 core)"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": f"{n} time steps from cold start ({el:.1f} s)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "jcg_iters_per_step": float(np.mean(its)),
    }
    print(json.dumps(line), flush=True)


PATHS = {
    # name: (bind mode, description)
    "plain": (0, "plain FP64 (reference arithmetic)"),
    "chosen": (8 | 16, "FP32 SpMV matrix + FP32 momentum element terms, FP64 assembly, "
                       "dot products, norms, stopping test and state"),
    "mixed": (1, "FP32 GWCE assembly + SpMV matrix + momentum, FP64 reductions and state"),
}


def _timed(gpu, it, W, K, dist):
    """W untimed steps, then K steps replayed as one graph, device-timed."""
    import torch
    if W > 0:
        gpu.run(it, W)
        it += W
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = gpu.launches()
    numitr, _ = gpu.run(it, K)
    torch.cuda.synchronize()
    it += K
    ms = gpu.last_run_ms()
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return it, ms, np.asarray(numitr), gpu.launches() - l0


def _accuracy(a, ref):
    """max |d eta|, RMS |d u| and wet/dry mismatches of state `a` against `ref`."""
    d = np.abs(a["eta2"] - ref["eta2"])
    both = (a["nodecode"] == 1) & (ref["nodecode"] == 1)
    mm = a["nodecode"] != ref["nodecode"]
    du = np.sqrt(np.mean((a["uu2"] - ref["uu2"]) ** 2 + (a["vv2"] - ref["vv2"]) ** 2))
    return {"max_deta_m": float(d.max()),
            "max_deta_both_wet_m": float(d[both].max()) if both.any() else 0.0,
            "p99_deta_m": float(np.percentile(d, 99)),
            "rms_du_ms": float(du), "wetdry_mismatch": int(mm.sum())}


def bench_gpu(args, rank, world, dist):
    import torch
    from adcirc_b200 import build, model, _lib
    build.build()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    case = make_case(args.case)
    cpu_case = case.clone() if (rank == 0 and world == 1 and not args.no_cpu) else None
    dt = case.params["dt"]
    W, K = args.warmup, args.steps
    names = ["chosen", "plain"] + ([] if args.no_mixed else ["mixed"])
    cases = {n: case.clone() for n in names}
    models = {n: model.GpuModel(cases[n], prec=PATHS[n][0]) for n in names}
    its = {n: 1 for n in names}
    res = {}
    with ClockSampler(local) as clk:
        for n in names:
            its[n], ms, numitr, launches = _timed(models[n], its[n], W, K, dist)
            res[n] = {"value": world * sim_days_per_hour(K, dt, ms / 1000.0), "ms_per_step": ms / K,
                      "jcg_iters_per_step": float(numitr.mean()), "gpu_launches": int(launches),
                      "mode": PATHS[n][0], "arithmetic": PATHS[n][1]}
    gpu = models["chosen"]
    # per-phase device times and the JCG roofline of the chosen path
    n_ph = 20
    ph = {"shift": 0.0, "gwce": 0.0, "jcg": 0.0, "wetdry": 0.0, "momentum": 0.0}
    iters = []
    for n in names:   # every path advances the same steps
        for k in range(n_ph):
            o = models[n].step(its[n] + k)
            if n == "chosen":
                iters.append(o.numitr)
                for kk, vv in gpu.phase_times().items():
                    ph[kk] += vv / n_ph
        its[n] += n_ph
    # e2e through the per-step public call (host round trip every step)
    K2 = min(K, args.e2e_steps)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(K2):
        gpu.step(its["chosen"] + k)
    el = time.perf_counter() - t0
    for n in names:
        if n != "chosen":
            models[n].run(its[n], K2)
        its[n] += K2
    if dist:
        t = torch.tensor([el], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        el = float(t.item())
    e2e = world * sim_days_per_hour(K2, dt, el)
    # accuracy of the FP32 paths against the FP64 path at hourly outputs
    acc = {n: [] for n in names if n != "plain"}
    hours = []
    spd = int(round(3600.0 / dt))
    for h in range(1, args.accuracy_hours + 1):
        target = h * spd + 1          # next step to run once hour h is complete
        if target <= its["plain"]:
            continue
        for n in names:
            models[n].run(its[n], target - its[n])
            its[n] = target
            models[n].sync_to_host()
        hours.append(h)
        for n in acc:
            acc[n].append(_accuracy(cases[n].arrays, cases["plain"].arrays))
    a = case.arrays
    nnz_o = int((a["nneigh"] - 1).sum())
    npn = case.sizes["np"]
    mean_it = float(np.mean(iters))
    peak, peak_kind = _peaks()
    achieved = (jcg_bytes(nnz_o, npn, mean_it, vbytes=4) / (ph["jcg"] / 1000.0) / 1e9
                if ph["jcg"] > 0 else 0.0)
    worst = {n: {k: max(x[k] for x in v) for k in v[0]} if v else None for n, v in acc.items()}
    line = {
        "metric": METRIC, "value": res["chosen"]["value"], "unit": UNIT, "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": res["chosen"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64+f32", "data": "synthetic",
        "config": {"workload": f"{args.case}: {npn} nodes, {case.sizes['ne']} elements, dt {dt} s, "
                               f"M2+K1 tides, {forcing(case)}, wet/dry on",
                   "path": "chosen: " + PATHS["chosen"][1],
                   "nodes": npn, "elements": case.sizes["ne"], "parallelism": f"replicas x{world}",
                   "l2": "resident state ~0.35 GB > 126 MB L2 (no flush)",
                   "first_step": 1 + W},
        "speedup_vs_plain_fp64": res["chosen"]["value"] / res["plain"]["value"],
        "paths": res,
        "accuracy_vs_fp64": {"hours": hours, "worst": worst, "per_hour": acc},
        "jcg_iters_per_step": res["chosen"]["jcg_iters_per_step"],
        "phase_ms": ph,
        "roofline": {"bound": "hbm", "kernel": "jcg_kernel", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": profiled_traffic(),
                     "traffic_source": "profiles/surge_kernels_full.md (ncu, one launch of "
                                       "jcg_kernel<1, float>, DRAM bytes read + written)",
                     "peak_kind": peak_kind, "iters_per_launch": mean_it},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 44, "d2h_bytes_per_step": 56,
                "steps": K2, "api": "adc_timestep per step"},
        "gpu_launches": res["chosen"]["gpu_launches"],
        "clocks": clk.summary(),
    }
    if cpu_case is not None:
        n, el_c, its_c = run_cpu_baseline(cpu_case, max_seconds=args.cpu_seconds)
        line["cpu_baseline"] = {"value": sim_days_per_hour(n, dt, el_c), "unit": UNIT, "cores": 1,
                                "kind": "port",
                                "sample": f"{n} time steps of the same mesh from cold start ({el_c:.1f} s)"}
    for m in models.values():
        m.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="adcgpu", choices=["adcgpu", "reference"])
    ap.add_argument("--case", default="surge", choices=["surge", "channel"])
    ap.add_argument("--accuracy-hours", type=int, default=3,
                    help="hourly outputs at which the FP32 paths are compared with FP64")
    ap.add_argument("--no-mixed", action="store_true", help="skip the all-FP32-assembly path")
    ap.add_argument("--e2e-steps", type=int, default=500)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as td
        backend = "nccl" if args.impl == "adcgpu" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        dist = td
    try:
        if args.impl == "reference":
            bench_reference(args, rank, world)
        else:
            bench_gpu(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
