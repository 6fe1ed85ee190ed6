"""Benchmark of the residual-and-update path on the 15 degree compression ramp.

Workload (the configuration the headline metric is quoted on): 400 x 200 quads split into 160,000
triangles, interior nodes jittered +-10% (numpy default_rng(0)), M = 2.5, p = 1e5 Pa, T = 300 K, AUSM flux,
second order with the Venkatakrishnan limiter K = 5, DPLUR with 4 sweeps, CFL 5, plain FP64. The mesh is
generated here (synthetic, deterministic). A step is one DPLUR iteration over the whole mesh (residual,
implicit operator, 4 sweeps, update); the metric is cell-updates/s (one residual evaluation + state update
of one cell).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl csu|reference]

The default line also carries `serve`: the serving headline (converged solves/hr of the continuous-batching
server with FP32 DPLUR blocks against the plain FP64 path one solve at a time, p50/p99 time-to-converge,
converged-state and force-coefficient differences) on a bounded seeded stream (csu_b200.servebench);
`--serve` runs a larger stream alone.

N > 1 (one process per GPU under torch.distributed.run) runs independent replicas of the solve, one per
GPU: the path has no exchange step at this size, so there is no collective in the timed region (weak
scaling). `--impl reference` times the reference solver compiled from its own C sources
(oracle/_ref, OpenMP on all host cores) on the same case and prints the same JSON line.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"
# CFL 10 (the configuration as first specified) diverges in the reference solver itself at iteration 90
# on this mesh (DPLUR with a global time step and 4 Jacobi sweeps); CFL 5 is stable.
CFL = 5.0
WORKLOAD = "ramp15_400x200_tri_dplur4_cfl5_ausm_fp64"


def workload_config(nc, nf, world):
    """The `config` object both arms print (the same keys, so the two lines name the same workload)."""
    return {"workload": WORKLOAD, "cells": nc, "faces": nf, "timestep": "DPLUR, 4 sweeps",
            "parallelism": "replicas%d" % world, "l2": "inputs larger than L2 (working set > 126 MB)"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def make_case(threads, tag):
    from csu_b200 import meshgen
    wd = "/tmp/csu_bench_%s/" % tag
    su2, inp = meshgen.ramp(threads=threads, cfl=CFL)
    if not os.path.exists(wd + "mesh.su2") or os.path.getsize(wd + "mesh.su2") != len(su2):
        meshgen.write_case(wd, su2, inp)
    else:
        with open(wd + "input.dat", "w") as f:
            f.write(inp)
    return wd


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
            "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
            "clocks_event_reasons.sw_power_cap"
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # start timing only once the sampler runs (its start-up must not fall inside the timed region)
            t0 = time.time()
            while not self.samples and time.time() - t0 < 5.0:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for n, v in zip(names, s[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def alg_bytes(case):
    """Compulsory bytes per launch of each kernel kind for this mesh (FP64 state, int32 indices):
    every array element the kernel needs is counted once, however often it is gathered."""
    nc, nf, nb = case.n_cells, case.n_faces, case.n_bfaces
    slots = int(case.cell_npts.sum())
    nint = 2 * nf
    W = 40                      # r u v p + T
    G = 96                      # gradient x, y and limiter of r u v p
    return {
        # W, npts, omega, x87 LSQ constants (a b c det + reciprocal), nei + dx dy + edge vectors per slot,
        # ghost geometry per boundary face, gradients/limiter out
        "grad": nc * (W + 4 + 8 + 56 + G) + slots * (4 + 16 + 16) + nb * 28,
        # face index/normal/|dS|/two centre offsets + flux out; boundary face data + flux out; cell W and G in
        "flux": nf * (8 + 16 + 8 + 32 + 32) + nb * (4 + 4 + 16 + 8 + 32) + nc * (W + G),
        # DPLUR diagonal (k_impl without R): W, counts, omega; per slot fslot; face cells, normal, |dS|;
        # boundary normal, |dS|; Omega/Lc and diagonal out
        "impl": nc * (W + 8 + 8 + 8 + 8) + slots * 4 + nf * 32 + nb * 24,
        # U and W of every cell (as a neighbour), counts; face cells, normal, |dS|; per interior slot fslot +
        # the 16 FP64 block out
        "blocks": nc * (32 + W + 4) + nf * 32 + nint * (4 + 128),
        # mean of the four sweeps of an iteration: x in, x out, counts, R, diagonal part, omega; per interior
        # slot its neighbour + 16 FP64 block; the first sweep also reads W, the face fluxes and the slots
        # (R gather), the last reads and writes U and writes W
        "sweep": nc * (32 + 32 + 4 + 32 + 8 + 8) + nint * (4 + 128)
                 + (nc * W + (nf + nb) * 32 + slots * 4 + nc * (32 + 32 + W)) // 4,
    }


def max_over_ranks(ms, dist, device):
    """The job's time: the slowest rank's. Every rank takes part in the same all-reduce (no-op alone)."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(cells, steps, world, ms):
    """Cell-updates per second of the whole job: every replica advances its own mesh `steps` times."""
    return cells * steps * world / (ms / 1e3)


def run_reference(wd, steps, warmup):
    """The reference's own solver functions (oracle/_ref), OpenMP on all host cores."""
    from oracle.refharness import Ref, available
    if not available():
        return None
    ref = Ref(wd)
    ref.iterate(max(warmup, 1))
    t0 = time.perf_counter()
    ref.iterate(steps)
    dt = time.perf_counter() - t0
    return ref.nc, ref.nf, dt


def reference_arm(args, rank):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    wd = make_case(threads, "ref")
    r = run_reference(wd, args.steps, args.warmup)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing"}))
        return 0
    nc, nf, dt = r
    v = nc * args.steps / dt
    line = {"metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(nc, nf, args.gpus),
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "reference",
                             "sample": "%d DPLUR iterations of the full 160k-cell ramp" % args.steps},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


SERVE_DEFAULT = {"n": 24, "cells_hi": 6e4, "rate": 20.0}


def serve_summary(n, cells_hi, rate):
    """The serving comparison of csu_b200.servebench on a bounded stream, summarized for the bench line."""
    from csu_b200 import servebench
    t0 = time.perf_counter()
    out = servebench.run(n=n, cells_hi=cells_hi, rate=rate)
    b, p = out["batched"], out["plain"]
    keys = ("solves_per_hour", "converged", "requests", "failed", "p50_s", "p99_s", "makespan_s",
            "cell_updates_per_s")
    def ratio(x, y):
        return x / y if x and y else None

    return {"metric": "converged solves/hr", "unit": "solves/hr",
            "vs_plain_fp64": ratio(b["solves_per_hour"], p["solves_per_hour"]),
            # time-to-converge of the plain arm over the batched arm's (higher is better for the batched arm)
            "p50_plain_over_batched": ratio(p["p50_s"], b["p50_s"]),
            "p99_plain_over_batched": ratio(p["p99_s"], b["p99_s"]),
            "batched_mixed": {k: b[k] for k in keys}, "plain_fp64": {k: p[k] for k in keys},
            "state_diff_rel": out["state_diff_rel"], "force_coef_diff_rel": out["coef_diff_rel"],
            "workload": out["workload"], "wall_s": time.perf_counter() - t0}


def airfoil_arm(args):
    """Batched transonic SST airfoils (csu_b200.airfoilbench): one pack of many C-meshes, FP32 DPLUR blocks
    against FP64 blocks, per-instance Cl/Cd differences."""
    import torch
    torch.cuda.set_device(0)
    from csu_b200 import airfoilbench
    out = airfoilbench.run(n=args.instances, ncells=args.instance_cells, iters=args.steps)
    line = {"metric": "cell-updates/s", "value": out["fp32"]["cell_updates_per_s"], "unit": "cell-updates/s",
            "n_gpus": 1, "steps": args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 residual, f32 DPLUR blocks", "data": "synthetic",
            "config": dict(out["workload"], workload="batched SST airfoils"), "result": out}
    print(json.dumps(line))
    return 0


def serve_arm(args):
    """Serving stream (csu_b200.servebench): requests of four geometry families arriving as a Poisson stream,
    served by the continuous-batching server (packs, FP32 DPLUR blocks) and by the plain FP64 path one solve
    at a time; metric: converged solves per hour of the batched server."""
    import torch
    torch.cuda.set_device(0)
    from csu_b200 import servebench
    out = servebench.run(n=args.requests, cells_hi=args.cells_hi, rate=args.rate)
    b, p = out["batched"], out["plain"]
    line = {"metric": "converged solves/hr", "value": b["solves_per_hour"], "unit": "solves/hr", "n_gpus": 1,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 residual, f32 DPLUR",
            "data": "synthetic", "config": dict(out["workload"], workload="serving stream"),
            "p50_s": b["p50_s"], "p99_s": b["p99_s"], "cell_updates_per_s": b["cell_updates_per_s"],
            "vs_plain_fp64": b["solves_per_hour"] / p["solves_per_hour"] if p["solves_per_hour"] else None,
            "plain_fp64": p, "batched": b, "state_diff_rel": out["state_diff_rel"],
            "iters": out["iters_batched"]}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="csu", choices=["csu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve", action="store_true",
                    help="the serving stream instead: batched mixed precision vs plain FP64, one solve at a time")
    ap.add_argument("--requests", type=int, default=40)
    ap.add_argument("--cells-hi", type=float, default=2e5)
    ap.add_argument("--rate", type=float, default=5.0, help="serving stream: Poisson arrivals per second")
    ap.add_argument("--airfoils", action="store_true",
                    help="the batched SST airfoil pack instead (FP32 vs FP64 DPLUR blocks, Cl/Cd differences)")
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--instance-cells", type=int, default=65536)
    ap.add_argument("--no-serve", action="store_true",
                    help="leave the bounded serving comparison out of the default line")
    args = ap.parse_args()
    if args.serve:
        return serve_arm(args)
    if args.airfoils:
        return airfoil_arm(args)
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import csu_b200
    wd = make_case(8, "r%d" % rank)
    case = csu_b200.Case.load(wd)
    eng = csu_b200.Engine(case)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    nc = case.n_cells

    # warm-up: the first call also captures the context's iteration graphs (8, 4, 2 and 1 iterations), so
    # the timed call of any length replays graphs only; the launch shapes the autotuner chose for this mesh
    # (faces per flux block, cells per sweep block) are read here, and a second warm-up recaptures the graphs
    # if that timing changed them
    eng.iterate(args.warmup)
    shapes = eng.autotune()
    eng.iterate(args.warmup, it0=args.warmup)
    torch.cuda.synchronize()
    launches0 = eng.stats()["kernel_launches"]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        eng.iterate(args.steps, it0=2 * args.warmup)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = eng.stats()["kernel_launches"] - launches0
    ws_mb = eng.stats()["device_bytes"] / 1e6
    ms = max_over_ranks(ms, dist, "cuda")
    if dist:
        dist.barrier()
    value = job_throughput(nc, args.steps, world, ms)

    # per-kernel device times of a few iterations, for the roofline of the dominant kernel
    kt = eng.time_kernels(5)
    names = ["prim", "grad", "flux", "rk", "impl", "sweep", "finalize", "resid", "blocks"]
    per = {n: (kt["ms"][i] / kt["count"][i] if kt["count"][i] else 0.0) for i, n in enumerate(names)}
    share = {n: kt["ms"][i] for i, n in enumerate(names)}
    dom = max(("grad", "flux", "impl", "sweep", "blocks"), key=lambda n: share[n])
    ab = alg_bytes(case)
    peak, peak_kind = peaks()
    achieved = ab[dom] / (per[dom] * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(dom)

    # end to end through the C ABI with host buffers: upload the state from pinned memory, one iteration,
    # read the state back, every step
    U = eng.get_state()
    pin = torch.empty(U.shape, dtype=torch.float64).pin_memory()
    host = pin.numpy()
    host[:] = U
    e2e_steps = max(10, args.steps // 10)
    for i in range(args.warmup):
        eng.set_state(host)
        eng.iterate(1, it0=i)
        eng.get_state(out=host)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        eng.set_state(host)
        eng.iterate(1, it0=i)
        eng.get_state(out=host)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e = nc * e2e_steps * world / e2e_s
    h2d = d2h = host.nbytes

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.refharness import available
        if available():
            threads = os.cpu_count() or 1
            wdr = make_case(threads, "cpu")
            r0 = run_reference(wdr, 2, 1)
            n_it = int(min(200, max(3, 15.0 / (r0[2] / 2))))
            nc_r, _, dt_r = run_reference(wdr, n_it, 1)
            cpu = {"value": nc_r * n_it / dt_r, "unit": METRIC, "cores": threads, "kind": "reference",
                   "sample": "%d DPLUR iterations of the full 160k-cell ramp (%.1f s)" % (n_it, dt_r)}

    # the serving headline (converged solves/hr, batched mixed precision vs plain FP64 one solve at a time)
    # on a bounded stream, after the timed region
    serve = None
    if rank == 0 and world == 1 and not args.no_serve:
        eng.close()
        eng = None
        serve = serve_summary(**SERVE_DEFAULT)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": workload_config(nc, case.n_faces, world),
                "working_set_mb": ws_mb, "launch_shapes": {"flux_faces_per_block": shapes[0],
                                                           "sweep_cells_per_block": shapes[1]},
                "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                             "alg_bytes_per_launch": ab[dom], "ms_per_launch": per[dom]},
                "kernel_ms_per_launch": per,
                "kernel_ms_share": {n: share[n] / max(sum(share.values()), 1e-30) for n in names},
                "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": launches, "clocks": clk.summary(), "cpu_baseline": cpu, "serve": serve}
        print(json.dumps(line))
    if eng is not None:
        eng.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
