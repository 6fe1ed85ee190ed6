"""Serving benchmark: a seeded stream of steady-solve requests on one GPU, served two ways.

  plain    one solve at a time in arrival order, FP64 DPLUR blocks (the plain single-solve GPU path)
  batched  the continuous-batching server (csu_srv_*): packs of concurrent solves, one launch per kernel
           per iteration for all of them, FP32 DPLUR blocks (mixed precision: the residual stays FP64)

Requests: geometry uniform over {channel with a 10 %-height bump, 15 deg wedge ramp, cylinder r = 0.5 in a
40-diameter box, NACA 0012 C-mesh}; cells log-uniform in [cells_lo, cells_hi]; M ~ U[0.3, 3] (at most 0.85
for the airfoil; at least 1.2 for the supersonic ramp); inviscid by default (`viscous=True` makes half of
them laminar, Re log-uniform in [1e3, 1e5]: many of those diverge with the explicit-diagonal DPLUR at these
settings, in both arms alike); local time steps at CFL 4; Poisson arrivals at `rate`
per second (numpy default_rng(seed)). Every solve is first order (AUSMDV) and stops at a residual drop
`drop` of the RMS density residual or after `max_iters` iterations. Reported per arm: solves per hour
(converged solves / makespan), p50 / p99 time-to-converge (finish - arrival), cell-updates/s; and the
largest difference between the two arms' converged states, relative to each variable's range.
"""
import math
import time

import numpy as np

from . import Case, Engine, Server, meshgen


def requests(n, seed=0, rate=5.0, cells_lo=1e4, cells_hi=2e5, viscous=False):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    out = []
    for k in range(n):
        geo = ["bump", "ramp", "cylinder", "airfoil"][int(rng.integers(4))]
        cells = int(math.exp(rng.uniform(math.log(cells_lo), math.log(cells_hi))))
        mach = float(rng.uniform(0.3, 3.0))
        if geo == "airfoil":
            mach = min(mach, 0.85)
        laminar = bool(rng.random() < 0.5) and viscous
        re = float(math.exp(rng.uniform(math.log(1e3), math.log(1e5)))) if laminar else None
        alpha = float(rng.uniform(-4.0, 4.0)) if geo == "airfoil" else 0.0
        out.append({"t": float(t[k]), "geo": geo, "cells": cells, "mach": mach, "laminar": laminar, "re": re,
                    "alpha": alpha})
    return out


def build_case(r, drop, fp32):
    viscous = "laminar" if r["laminar"] else None
    solver = {"order": 1, "cfl": 5.0, "flux": "AUSMDV"}
    if r["geo"] == "bump":
        su2, inp = meshgen.bump(ncells=r["cells"], mach=r["mach"], viscous=viscous, re=r["re"], **solver)
    elif r["geo"] == "cylinder":
        su2, inp = meshgen.cylinder(ncells=r["cells"], mach=max(r["mach"], 0.3), viscous=viscous, re=r["re"],
                                    **solver)
    elif r["geo"] == "airfoil":
        su2, inp = meshgen.airfoil(ncells=r["cells"], mach=r["mach"], alpha_deg=r["alpha"], y1=1e-4,
                                   viscous=viscous, re=r["re"], **solver)
    else:
        nj = max(4, int(round(math.sqrt(r["cells"] / 4.0))))
        mach = max(r["mach"], 1.2)
        p = meshgen._pressure_for_re(r["re"], mach, 300.0, 1.5) if viscous else 1e5
        su2, inp = meshgen.ramp(ni=2 * nj, nj=nj, mach=mach, pressure=p, flux="AUSMDV", order=1, cfl=5.0)
        if viscous:
            inp += "laminar, 1\n"
    # local time steps (CFL 4): the global step of the reference is set by the smallest cell and barely
    # moves the stretched airfoil and cylinder grids
    inp += "convDrop, %g\nimplicitFP32, %d\nimplicitLocalDt, 1\nCFL, 4.0\n" % (drop, 1 if fp32 else 0)
    return Case.from_text(inp, su2)


def _pct(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def run_plain(reqs, cases, max_iters):
    """One solve at a time in arrival order; a solve starts at max(its arrival, the previous finish)."""
    t0 = time.perf_counter()
    res, states, cu = [], [], 0
    for r, case in zip(reqs, cases):
        now = time.perf_counter() - t0
        if now < r["t"]:
            time.sleep(r["t"] - now)
        eng = Engine(case)
        failed = False
        try:
            done = len(eng.iterate_until(max_iters))
        except Exception:
            done, failed = max_iters, True
        states.append(eng.get_state())
        cu += case.n_cells * done
        eng.close()
        res.append({"finish": time.perf_counter() - t0, "iters": done, "converged": done < max_iters and not failed,
                    "failed": failed})
    return res, states, cu, time.perf_counter() - t0


def run_batched(reqs, cases, max_iters, budget_bytes, iters_per_step=16, rebuild_steps=8, prep_threads=2):
    # meshes are prepared on background threads while the packs iterate
    srv = Server(budget_bytes, iters_per_step=iters_per_step, rebuild_steps=rebuild_steps,
                 prep_threads=prep_threads)
    t0 = time.perf_counter()
    ids = [None] * len(reqs)
    nxt = 0
    finished = {}
    while len(finished) < len(reqs):
        now = time.perf_counter() - t0
        while nxt < len(reqs) and reqs[nxt]["t"] <= now:
            ids[nxt] = srv.submit(cases[nxt], max_iters=max_iters)
            nxt += 1
        running, queued = srv.step()
        for k in range(nxt):
            if k in finished:
                continue
            info = srv.info(ids[k])
            if info["state"] in ("converged", "maxiter", "failed"):
                finished[k] = info
        if running == 0 and queued == 0 and nxt < len(reqs):
            time.sleep(max(0.0, reqs[nxt]["t"] - (time.perf_counter() - t0)))
    makespan = time.perf_counter() - t0
    res, states = [], []
    for k in range(len(reqs)):
        info = finished[k]
        states.append(srv.take(ids[k]))
        res.append({"finish": info["t_end"], "iters": info["iters"], "converged": info["state"] == "converged",
                    "failed": info["state"] == "failed"})
    tot = srv.totals()
    srv.close()
    run_batched.last_totals = tot
    return res, states, tot["cell_updates"], makespan


def summarize(reqs, res, cu, makespan):
    lat = [x["finish"] - r["t"] for r, x in zip(reqs, res) if x["converged"]]
    n_conv = sum(1 for x in res if x["converged"])
    n_fail = sum(1 for x in res if x.get("failed"))
    return {"solves_per_hour": n_conv / makespan * 3600.0, "converged": n_conv, "failed": n_fail,
            "requests": len(res),
            "p50_s": _pct(lat, 50), "p99_s": _pct(lat, 99), "makespan_s": makespan,
            "cell_updates_per_s": cu / makespan}


def state_difference(a, b):
    """Largest |a - b| over all cells, relative to each variable's range in b."""
    worst = 0.0
    for x, y in zip(a, b):
        rng = np.maximum(np.ptp(y, axis=1, keepdims=True), np.abs(y).max(axis=1, keepdims=True) * 1e-12)
        worst = max(worst, float(np.max(np.abs(x - y) / rng)))
    return worst


def run(n=40, seed=0, rate=5.0, cells_lo=1e4, cells_hi=2e5, drop=1e-8, max_iters=3000, budget_gb=150.0,
        viscous=False):
    reqs = requests(n, seed, rate, cells_lo, cells_hi, viscous)
    plain_cases = [build_case(r, drop, False) for r in reqs]
    batched_cases = [build_case(r, drop, True) for r in reqs]
    pr, ps, pcu, pt = run_plain(reqs, plain_cases, max_iters)
    br, bs, bcu, bt = run_batched(reqs, batched_cases, max_iters, int(budget_gb * (1 << 30)))
    plain = summarize(reqs, pr, pcu, pt)
    batched = summarize(reqs, br, bcu, bt)
    both = [k for k in range(n) if pr[k]["converged"] and br[k]["converged"]]
    diff = state_difference([bs[k] for k in both], [ps[k] for k in both]) if both else None
    batched["server"] = getattr(run_batched, "last_totals", None)
    return {"plain": plain, "batched": batched, "state_diff_rel": diff,
            "iters_plain": [x["iters"] for x in pr], "iters_batched": [x["iters"] for x in br],
            "workload": {"requests": n, "seed": seed, "rate_per_s": rate, "cells": [cells_lo, cells_hi],
                         "drop": drop, "max_iters": max_iters, "order": 1, "flux": "AUSMDV", "viscous": viscous,
                         "time_step": "local, CFL 4",
                         "geometries": ["bump", "ramp", "cylinder", "airfoil"]}}
