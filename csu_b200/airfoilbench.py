"""Batched transonic airfoils: many SST solves advanced by one launch per kernel, FP32 DPLUR blocks against FP64.

Workload (the batched-airfoil configuration): `n` NACA 0012 C-meshes (closed trailing edge, 512 x 128 quads
for 65,536 cells by default, first cell 1e-6 chord, far field at 100 chords; csu_b200.meshgen.airfoil), each
with its own Mach number M ~ U[0.5, 0.85] and angle of attack alpha ~ U[-4, 4] deg from numpy
default_rng(seed), Re = 6e6 on the chord, Menter SST. All solves form one pack (csu_pack_*): every kernel
of an iteration is one launch for all of them, replayed from CUDA graphs. Solver settings: first order, AUSM,
DPLUR with local time steps (an extension: the reference's SST DPLUR is undefined), the destruction part of
the SST source Jacobians in the diagonal, CFL ramped geometrically from `cfl0` to `cfl1` over `ramp` iterations.

Two packs of the same solves run the same number of iterations: FP64 blocks and FP32 blocks (the residual,
the state and the sweeps' accumulation stay FP64 in both). Reported: per-instance lift and drag coefficients
from the body-axis force coefficients of solverCalcCoeff3 (solver.c:1342-1401) rotated by alpha,
Cl = -Cx sin(alpha) + Cy cos(alpha), Cd = Cx cos(alpha) + Cy sin(alpha); their difference between the
precisions; residual drops; cell-updates per second of each pack.
"""
import math
import time

import numpy as np

from . import Case, Pack, Prep, meshgen


def instances(n=64, seed=0):
    rng = np.random.default_rng(seed)
    return [{"mach": float(rng.uniform(0.5, 0.85)), "alpha": float(rng.uniform(-4.0, 4.0))} for _ in range(n)]


def build(inst, ncells, fp32, cfl0, cfl1, ramp, n_linear, mesh_cache):
    key = ncells
    if key not in mesh_cache:
        # the mesh is the same for every instance; only the flow conditions differ
        mesh_cache[key] = meshgen.airfoil(ncells=ncells, mach=0.7, alpha_deg=0.0, y1=1e-6, far=100.0,
                                          viscous="sst", re=6e6, flux="AUSM", order=1, n_linear=n_linear,
                                          cfl=cfl0)[0]
    su2 = mesh_cache[key]
    _, inp = meshgen.airfoil(ncells=64, mach=inst["mach"], alpha_deg=inst["alpha"], y1=1e-6, far=100.0,
                             viscous="sst", re=6e6, flux="AUSM", order=1, n_linear=n_linear, cfl=cfl0)
    inp += "implicitLocalDt, 1\nimplicitFP32, %d\nCFLramp, %d\nCFLmax, %g\n" % (1 if fp32 else 0, ramp, cfl1)
    return Case.from_text(inp, su2)


def lift_drag(coef, alpha_deg):
    a = math.radians(alpha_deg)
    cx, cy = coef[0] + coef[1], coef[2] + coef[3]
    return -cx * math.sin(a) + cy * math.cos(a), cx * math.cos(a) + cy * math.sin(a)


def run_pack(insts, ncells, fp32, iters, cfl0, cfl1, ramp, n_linear, mesh_cache):
    cases = [build(i, ncells, fp32, cfl0, cfl1, ramp, n_linear, mesh_cache) for i in insts]
    preps = [Prep(c) for c in cases]
    pack = Pack(preps)
    cells = sum(c.n_cells for c in cases)
    t0 = time.perf_counter()
    pack.iterate(iters)
    infos = [pack.info(k) for k in range(len(preps))]  # waits for the iterations
    dt = time.perf_counter() - t0
    out = []
    for inst, info in zip(insts, infos):
        cl, cd = lift_drag(info["coef"], inst["alpha"])
        drop = float(info["res"][0] / info["res0"][0]) if info["have_res0"] and info["res0"][0] > 0 else None
        out.append({"cl": cl, "cd": cd, "iter": info["iter"], "status": info["status"], "drop": drop})
    bytes_ = pack.stats()["device_bytes"]
    pack.close()
    return out, {"seconds": dt, "cells": cells, "cell_updates_per_s": cells * iters / dt, "device_bytes": bytes_}


def run(n=64, ncells=65536, iters=2000, seed=0, cfl0=2.0, cfl1=16.0, ramp=300, n_linear=16):
    insts = instances(n, seed)
    cache = {}
    r32, p32 = run_pack(insts, ncells, True, iters, cfl0, cfl1, ramp, n_linear, cache)
    r64, p64 = run_pack(insts, ncells, False, iters, cfl0, cfl1, ramp, n_linear, cache)
    dcl = [abs(a["cl"] - b["cl"]) for a, b in zip(r32, r64)]
    dcd = [abs(a["cd"] - b["cd"]) for a, b in zip(r32, r64)]
    ok = [a["status"] == 0 and b["status"] == 0 for a, b in zip(r32, r64)]
    return {"workload": {"instances": n, "cells_per_instance": ncells, "iterations": iters, "seed": seed,
                         "model": "SST", "flux": "AUSM", "order": 1, "re": 6e6, "y1": 1e-6,
                         "time_step": "DPLUR %d sweeps, local steps, CFL %g -> %g over %d" % (n_linear, cfl0, cfl1,
                                                                                              ramp)},
            "fp32": p32, "fp64": p64, "speedup_fp32_blocks": p32["cell_updates_per_s"] / p64["cell_updates_per_s"],
            "finite_both": int(sum(ok)),
            "cl_abs_diff_max": max(d for d, o in zip(dcl, ok) if o) if any(ok) else None,
            "cd_abs_diff_max": max(d for d, o in zip(dcd, ok) if o) if any(ok) else None,
            "cl_rel_diff_max": max(d / max(abs(b["cl"]), 1e-12) for d, b, o in zip(dcl, r64, ok) if o) if any(ok) else None,
            "cd_rel_diff_max": max(d / max(abs(b["cd"]), 1e-12) for d, b, o in zip(dcd, r64, ok) if o) if any(ok) else None,
            "drop_fp64_median": float(np.median([b["drop"] for b, o in zip(r64, ok) if o])) if any(ok) else None,
            "instances_detail": [{"mach": i["mach"], "alpha": i["alpha"], "cl64": b["cl"], "cd64": b["cd"],
                                  "cl32": a["cl"], "cd32": a["cd"], "drop64": b["drop"], "drop32": a["drop"],
                                  "status64": b["status"], "status32": a["status"]}
                                 for i, a, b in zip(insts, r32, r64)]}
