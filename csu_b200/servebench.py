"""Serving benchmark: a seeded stream of steady-solve requests on one GPU, served two ways.

  plain    one solve at a time in arrival order, FP64 DPLUR blocks (the plain single-solve GPU path)
  batched  the continuous-batching server (csu_srv_*): packs of concurrent solves, one launch per kernel
           per iteration for all of them, FP32 DPLUR blocks (mixed precision: the residual stays FP64)

Requests (the serving configuration): geometry uniform over `families` (channel with a 10 %-height bump,
15 deg wedge ramp, cylinder r = 0.5 in a 40-diameter box, NACA 0012 C-mesh); cells log-uniform in
[cells_lo, cells_hi]; M ~ U[0.3, 3] (at most 0.85 for the airfoil; at least 1.2 for the ramp, a supersonic
inflow); half laminar with Re log-uniform in [1e3, 1e5], half Spalart-Allmaras with Re log-uniform in
[1e6, 1e7]; Poisson arrivals at `rate` per second; all from numpy default_rng(seed).

Solver settings, the same in both arms: first order, AUSM, DPLUR with 16 sweeps and local time steps at
CFL 16, stop at a residual drop `drop` of the RMS density residual (from its largest value so far) or after
`max_iters` iterations. AUSM
rather than AUSMDV: AUSMDV's switches leave the reference's own solution limit-cycling at 1e-5..1e-4 of the
initial residual on the cylinder (its LU-SGS at CFL 1000 as well), so no 1e-8 drop exists for it to reach;
AUSM converges the same case to 1e-13. The airfoil family is left out of the default stream: on its C-mesh
the residual of every scheme stalls near 0.2 of its initial value in the wake block (the reference's as
well), so its requests would only measure the iteration cap.

Reported per arm: solves per hour (converged solves / makespan), p50 / p99 time-to-converge (finish -
arrival) over converged requests, cell-updates/s, converged / failed counts; and between the arms, for
requests converged in both: the largest state difference relative to each variable's range, and the
largest difference of the force coefficients (Cx_p, Cx_v, Cy_p, Cy_v of the last iteration) relative to
the largest coefficient of that request.
"""
import math
import time

import numpy as np

from . import Case, Engine, Server, meshgen

FAMILIES = ("bump", "ramp", "cylinder")
ALL_FAMILIES = ("bump", "ramp", "cylinder", "airfoil")
SOLVER = {"flux": "AUSM", "order": 1, "n_linear": 16, "cfl": 16.0}


def requests(n, seed=0, rate=5.0, cells_lo=1e4, cells_hi=2e5, families=FAMILIES):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    out = []
    for k in range(n):
        geo = families[int(rng.integers(len(families)))]
        cells = int(math.exp(rng.uniform(math.log(cells_lo), math.log(cells_hi))))
        mach = float(rng.uniform(0.3, 3.0))
        if geo == "airfoil":
            mach = min(mach, 0.85)
        if geo == "ramp":
            mach = max(mach, 1.2)
        if rng.random() < 0.5:
            model, re = "laminar", float(math.exp(rng.uniform(math.log(1e3), math.log(1e5))))
        else:
            model, re = "sa", float(math.exp(rng.uniform(math.log(1e6), math.log(1e7))))
        alpha = float(rng.uniform(-4.0, 4.0)) if geo == "airfoil" else 0.0
        out.append({"t": float(t[k]), "geo": geo, "cells": cells, "mach": mach, "model": model, "re": re,
                    "alpha": alpha})
    return out


def build_case(r, drop, fp32):
    visc, re = r["model"], r["re"]
    solver = {"order": SOLVER["order"], "cfl": SOLVER["cfl"], "flux": SOLVER["flux"], "n_linear": SOLVER["n_linear"]}
    if r["geo"] == "bump":
        su2, inp = meshgen.bump(ncells=r["cells"], mach=r["mach"], viscous=visc, re=re, **solver)
    elif r["geo"] == "cylinder":
        su2, inp = meshgen.cylinder(ncells=r["cells"], mach=r["mach"], viscous=visc, re=re, **solver)
    elif r["geo"] == "airfoil":
        su2, inp = meshgen.airfoil(ncells=r["cells"], mach=r["mach"], alpha_deg=r["alpha"], y1=1e-5,
                                   viscous=visc, re=re, **solver)
    else:
        nj = max(4, int(round(math.sqrt(r["cells"] / 4.0))))
        p = meshgen._pressure_for_re(re, r["mach"], 300.0, 1.5)
        su2, inp = meshgen.ramp(ni=2 * nj, nj=nj, mach=r["mach"], pressure=p, flux=solver["flux"],
                                order=solver["order"], cfl=solver["cfl"], n_linear=solver["n_linear"])
        inp += "laminar, 1\n" if visc == "laminar" else "sa, 1\nturbRatio, 3\n"
    # local time steps: the global step of the reference is set by the smallest cell and barely moves the
    # stretched grids
    inp += "convDrop, %g\nimplicitFP32, %d\nimplicitLocalDt, 1\n" % (drop, 1 if fp32 else 0)
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
        coef = [0.0] * 4
        try:
            h = eng.iterate_until(max_iters)
            done = len(h)
            coef = [float(v) for v in h[-1, case.nvar:case.nvar + 4]]
        except Exception:
            done, failed = max_iters, True
        states.append(eng.get_state())
        cu += case.n_cells * done
        eng.close()
        res.append({"finish": time.perf_counter() - t0, "iters": done, "converged": done < max_iters and not failed,
                    "failed": failed, "coef": coef})
    return res, states, cu, time.perf_counter() - t0


def run_batched(reqs, cases, max_iters, budget_bytes, iters_per_step=16, rebuild_steps=8, prep_threads=2):
    # meshes are prepared on background threads while the packs iterate
    srv = Server(budget_bytes, iters_per_step=iters_per_step, rebuild_steps=rebuild_steps,
                 prep_threads=prep_threads)
    t0 = time.perf_counter()
    ids = [None] * len(reqs)
    index = {}
    nxt = 0
    finished = {}
    while len(finished) < len(reqs):
        now = time.perf_counter() - t0
        while nxt < len(reqs) and reqs[nxt]["t"] <= now:
            ids[nxt] = srv.submit(cases[nxt], max_iters=max_iters)
            index[ids[nxt]] = nxt
            nxt += 1
        running, queued = srv.step()
        for rid in srv.poll():
            finished[index[rid]] = srv.info(rid)
        if running == 0 and queued == 0 and nxt < len(reqs):
            time.sleep(max(0.0, reqs[nxt]["t"] - (time.perf_counter() - t0)))
    makespan = time.perf_counter() - t0
    res, states = [], []
    for k in range(len(reqs)):
        info = finished[k]
        states.append(srv.take(ids[k]))
        res.append({"finish": info["t_end"], "iters": info["iters"], "converged": info["state"] == "converged",
                    "failed": info["state"] == "failed", "coef": info["coef"]})
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


def coef_difference(a, b):
    """Largest |a - b| of the force coefficients over requests, relative to the largest |b| of each."""
    worst = 0.0
    for x, y in zip(a, b):
        x, y = np.asarray(x), np.asarray(y)
        worst = max(worst, float(np.max(np.abs(x - y)) / max(float(np.max(np.abs(y))), 1e-300)))
    return worst


def run(n=40, seed=0, rate=5.0, cells_lo=1e4, cells_hi=2e5, drop=1e-8, max_iters=20000, budget_gb=150.0,
        families=FAMILIES, iters_per_step=32, rebuild_steps=4):
    reqs = requests(n, seed, rate, cells_lo, cells_hi, families)
    plain_cases = [build_case(r, drop, False) for r in reqs]
    batched_cases = [build_case(r, drop, True) for r in reqs]
    pr, ps, pcu, pt = run_plain(reqs, plain_cases, max_iters)
    br, bs, bcu, bt = run_batched(reqs, batched_cases, max_iters, int(budget_gb * (1 << 30)),
                                  iters_per_step=iters_per_step, rebuild_steps=rebuild_steps)
    plain = summarize(reqs, pr, pcu, pt)
    batched = summarize(reqs, br, bcu, bt)
    both = [k for k in range(n) if pr[k]["converged"] and br[k]["converged"]]
    diff = state_difference([bs[k] for k in both], [ps[k] for k in both]) if both else None
    cdiff = coef_difference([br[k]["coef"] for k in both], [pr[k]["coef"] for k in both]) if both else None
    batched["server"] = getattr(run_batched, "last_totals", None)
    return {"plain": plain, "batched": batched, "state_diff_rel": diff, "coef_diff_rel": cdiff,
            "iters_plain": [x["iters"] for x in pr], "iters_batched": [x["iters"] for x in br],
            "workload": {"requests": n, "seed": seed, "rate_per_s": rate, "cells": [cells_lo, cells_hi],
                         "drop": drop, "max_iters": max_iters, "order": SOLVER["order"], "flux": SOLVER["flux"],
                         "models": "half laminar Re 1e3-1e5, half SA Re 1e6-1e7",
                         "time_step": "DPLUR %d sweeps, local steps, CFL %g" % (SOLVER["n_linear"], SOLVER["cfl"]),
                         "geometries": list(families)}}
