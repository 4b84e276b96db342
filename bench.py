#!/usr/bin/env python
"""Benchmark of the eikonal solve path: grid updates per second on the Riemann3 192^3 plain solve.

Workload: 192^3 grid on [0,1]^3, metric R diag(1, a1^-2, a2^-2) R^T (a1, a2 in [1,20], smooth
random rotation), 40 spherical walls (radii 0.02-0.08), 16 seeds (hamiltonfastmarching_b200.workloads
.riemann3_case, seed = 1 + rank). One step = one complete solve (Selling stencils, wall visibility,
tile dependency graph, fast-iterative solve) of the instance; a grid update is one reached cell
(the reference's nAccepted). Synthetic data; the 340 MB metric exceeds the 126 MB L2, so no flush
is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is measured with inputs resident in HBM through the device entry point of the C ABI;
`e2e` through the public HFMIO call with host arrays (host->device and device->host copies inside
the timed region). With --gpus N under torchrun every rank solves its own instance (replicas:
the path does not shard) and the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_UPDATE = {64: 57, 32: 53}  # metric 6x8 B + wall 1 B + value 8|4 B per reached cell
WORKLOAD = "Riemann3 192^3 plain solve, 40 spherical walls, 16 seeds"


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--side", type=int, default=192, help="grid side of the benchmarked instance")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-riemann", type=int, default=384, help="Riemann2 instances of the batched mix")
    ap.add_argument("--batch-lifted", type=int, default=128, help="ReedsShepp2/Elastica2 instances of the mix")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched mixed-model leg")
    ap.add_argument("--serve-rates", default="50,100,200,500,1000,2000",
                    help="Poisson arrival rates (req/s) of the serving leg")
    ap.add_argument("--serve-requests", type=int, default=300, help="requests per arrival rate")
    ap.add_argument("--serve-pool", type=int, default=48, help="distinct request payloads the arrivals draw from")
    ap.add_argument("--serve-resident", type=int, default=64, help="instances resident at once in the served arm")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--tti-side", type=int, default=128, help="grid side of the TTI3 differentiation leg")
    ap.add_argument("--tti-fd-voxels", type=int, default=32, help="voxels checked by central differences")
    ap.add_argument("--no-diff", action="store_true", help="skip the TTI3 differentiation leg")
    ap.add_argument("--geo-side", type=int, default=1024, help="grid side of the geodesic leg (Riemann2)")
    ap.add_argument("--geo-tips", type=int, default=4096, help="tips of the geodesic leg")
    ap.add_argument("--geo-cpu-tips", type=int, default=64, help="tips timed on the reference CPU build")
    ap.add_argument("--no-geo", action="store_true", help="skip the geodesic leg")
    return ap.parse_args(argv)


# ------------------------------------------------------------------------------------------ utils

def rank_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(key):
    """Per-launch DRAM bytes of the solver kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "fim_kernel_traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 2 and parts[0] == key:
                return float(parts[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region (every 200 ms)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.tmp, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.tmp.flush()
        rows = []
        with open(self.tmp.name) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def bench_config(n):
    """The workload description, identical in both arms of the benchmark."""
    return {"workload": WORKLOAD, "grid": [n, n, n], "generator": "workloads.riemann3_case(n, seed=1 + rank)",
            "instances_per_step": "one per rank", "precision": "f64", "l2": "inputs larger than L2 (340 MB metric)"}


def reference_cpu_sample(side, seed=1):
    """The reference's FileHFM_Riemann3 (built from its sources) on one full solve of the benchmarked
    instance: updates/s = nAccepted / (FMCPUTime + StencilCPUTime), one core."""
    from oracle.refrun import have_reference, run_reference
    from hamiltonfastmarching_b200 import workloads as W
    if not have_reference("Riemann3"):
        return None
    p = W.riemann3_case(side, seed=seed)
    p["exportValues"] = 0.0
    t0 = time.time()
    out = run_reference(p)
    wall = time.time() - t0
    if out.get("retcode") != 0:
        return None
    cpu_s = out["FMCPUTime"] + out["StencilCPUTime"]
    return {"value": out["nAccepted"] / cpu_s, "unit": "grid-updates/s", "cores": 1, "kind": "reference",
            "sample": f"FileHFM_Riemann3, one full solve of the benchmarked {side}^3 instance "
                      f"({int(out['nAccepted'])} reached cells): FMCPUTime {out['FMCPUTime']:.2f} s + "
                      f"StencilCPUTime {out['StencilCPUTime']:.2f} s (wall {wall:.1f} s incl. file IO)"}


# ------------------------------------------------------------------------------- batched leg

def batched_leg(args, rank, world):
    """Batched mixed-model launch vs the plain one-at-a-time GPU solve of the same instances.

    384 Riemann2 (sides log-uniform in [64,1024], anisotropy 1-10) + 128 lifted instances
    (ReedsShepp2 / Elastica2, N x N x 60, N log-uniform in [64,256], tubular-image cost), FP32.
    Both arms go through the public API from host arrays (hfm_run per store vs one hfm_run_batch
    over all stores); stores are filled before the timed region. The FP32 values of a seeded 5%
    sample are compared with the FP64 path (itself held to the reference at 1e-10 by the tests).
    """
    import hamiltonfastmarching_b200 as H
    from hamiltonfastmarching_b200 import workloads as W
    t0 = time.perf_counter()
    cases = W.batched_mix(args.batch_riemann, args.batch_lifted, seed=3 + rank,
                          processes=min(16, os.cpu_count() or 1))
    gen_s = time.perf_counter() - t0
    cells = int(sum(int(np.prod(p["dims"])) for p in cases))
    rng = np.random.default_rng(1234)
    sample = sorted(rng.choice(len(cases), max(1, len(cases) // 20), replace=False).tolist())
    sample_cases = {k: dict(cases[k], solverPrecision="float64", verbosity=0.0) for k in sample}
    ios = []
    for k in range(len(cases)):
        io = H.HFMIO("RowMajor")
        io.set_dict(cases[k], views=True)  # the store reads the case's arrays in place
        io.set_scalar("verbosity", 0)
        ios.append(io)

    def clear():
        for io in ios:
            if io.has_field("values"):
                io.erase_field("values")

    def batched():
        codes = H.run_ios(ios)
        if any(codes):
            raise RuntimeError(f"batched solve failed: {sorted(set(codes))}")

    def plain():
        for io in ios:
            io.run()

    batched()  # warm-up of both paths (allocator pool, module load)
    clear()
    plain()
    clear()
    out = {}
    for name, fn in (("batched", batched), ("plain", plain)):
        t0 = time.perf_counter()
        fn()
        el = time.perf_counter() - t0
        reached = sum(io.get_scalar("nAccepted") for io in ios)
        out[name] = {"seconds": el, "solves_per_s": len(ios) / el, "grid_updates_per_s": reached / el}
        if name == "batched":
            vals32 = {k: ios[k].get_array("values") for k in sample}
        clear()
    # autotuned schedule: per family, a coordinate search on its batch (GPU time of the family's
    # launch sequence), then the whole batched solve again with the tuned tile shape / sweeps / queue
    from hamiltonfastmarching_b200.autotune import Autotuner
    tuned = {}
    at = Autotuner(repeats=1)
    t0 = time.perf_counter()
    fams = {}
    for k in range(len(ios)):
        fams.setdefault(ios[k].get_string("model"), []).append(k)
    for fam, ks in fams.items():
        # on the family's own batch (the schedule is tuned for the batch it will run), over sweeps
        # and queue policy (tile shapes seldom win on these grids and double the search)
        tuned[fam] = at.tune([cases[k] for k in ks], sweeps=1, params=("tileSweeps", "queue"))
    tune_s = time.perf_counter() - t0
    for k, io in enumerate(ios):
        t = at.lookup(cases[k])
        io.set_scalar("tileSweeps", float(t["tileSweeps"]))
        io.set_array("tileShape", np.asarray(t["tileShape"], float))
        kind, lo, hi = t["queue"]
        io.set_scalar("tileOrdering", 1.0 if kind == "band" else 0.0)
        if kind == "band":
            io.set_scalar("bandLo", float(lo))
            io.set_scalar("bandHi", float(hi))
    batched()
    clear()
    t0 = time.perf_counter()
    batched()
    el = time.perf_counter() - t0
    reached = sum(io.get_scalar("nAccepted") for io in ios)
    out["batched_autotuned"] = {"seconds": el, "solves_per_s": len(ios) / el, "grid_updates_per_s": reached / el,
                                "tuning_s": tune_s,
                                "tuned": {f: {"tileShape": v["tileShape"], "tileSweeps": v["tileSweeps"],
                                              "queue": v["queue"], "sample_speedup": v["default_seconds"] / v["seconds"]}
                                          for f, v in tuned.items()}}
    clear()
    # FP64 on the sample
    errs = []
    res64 = H.run_batch([sample_cases[k] for k in sample])
    for k, r in zip(sample, res64):
        v64, v32 = r["values"], vals32[k]
        fin = np.isfinite(v64)
        errs.append(float(np.max(np.abs(v64[fin] - v32[fin])) / np.max(np.abs(v64[fin]))))
    return {"workload": f"{args.batch_riemann} Riemann2 (64-1024 sides) + {args.batch_lifted} ReedsShepp2/Elastica2 "
                        f"(N x N x 60, N 64-256), FP32, one hfm_run_batch",
            "instances": len(ios), "cells": cells,
            "batched": out["batched"], "plain_one_at_a_time": out["plain"],
            "batched_autotuned": out["batched_autotuned"],
            "speedup_solves_per_s": out["batched"]["solves_per_s"] / out["plain"]["solves_per_s"],
            "speedup_autotuned_solves_per_s": out["batched_autotuned"]["solves_per_s"] / out["plain"]["solves_per_s"],
            "fp32_max_rel_err_vs_fp64": max(errs), "fp64_sample": len(sample), "input_generation_s": gen_s,
            "path": "public API from host arrays (H2D/D2H inside both timings)"}


# ------------------------------------------------------------------------------- serving leg

def serving_leg(args, rank, world):
    """Continuous-batching server vs a plain one-at-a-time GPU solve loop on the same arrivals.

    Requests: 60% Riemann2 (64-1024 sides), 25% Riemann3 (64-192, walls), 15% ReedsShepp2
    (N x N x 60, N 64-256), 1-4 seeds, FP32, drawn from a pool of distinct seeded payloads;
    Poisson arrivals at each rate. The served arm is hfm_server with resident solvers (up to
    --serve-resident instances at once, each released when its own tiles converge); the plain arm
    is the same server with max_batch = 1 (every request through hfm_run, one at a time on the
    whole GPU). Latency = completion - submit (host clock of the server); throughput = requests /
    (last completion - first submit). Both arms run the same requests in the same order.
    """
    import threading
    import hamiltonfastmarching_b200 as H
    from hamiltonfastmarching_b200 import workloads as W
    from hamiltonfastmarching_b200.serving import Server
    t0 = time.perf_counter()
    specs = W.serving_specs(args.serve_pool, seed=5 + rank)
    pool = W.generate(specs, processes=min(16, os.cpu_count() or 1))
    for p in pool:
        p["solverPrecision"] = "float32"
        p["verbosity"] = 0.0
        p.pop("exportValues", None)
        p["exportValues"] = 1.0
    gen_s = time.perf_counter() - t0
    cells = [int(np.prod(p["dims"])) for p in pool]
    rates = [float(r) for r in args.serve_rates.split(",") if r]

    def run_arm(max_batch, rate, seed):
        rng = np.random.default_rng(seed)
        picks = rng.integers(0, len(pool), args.serve_requests)
        gaps = rng.exponential(1.0 / rate, args.serve_requests)
        tickets = [None] * args.serve_requests
        lat, done_t, sub_t, slow = [], [], [], []
        with Server(max_batch=max_batch) as srv:
            def waiter():
                for i in range(args.serve_requests):
                    while tickets[i] is None:
                        time.sleep(0.0005)
                    t = tickets[i]
                    t.wait()
                    if t.status != 0:
                        raise RuntimeError(f"request failed with status {t.status}")
                    sub_t.append(t.times[0])
                    done_t.append(t.times[2])
                    lat.append(t.latency)
                    slow.append((t.latency, i, t.times[1] - t.times[0]))
                    tickets[i] = False  # drop the store (and its outputs)
            th = threading.Thread(target=waiter)
            th.start()
            start = time.perf_counter()
            due = start
            for i in range(args.serve_requests):
                due += gaps[i]
                d = due - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets[i] = srv.submit(pool[picks[i]])
            th.join()
            st = srv.stats()
        span = max(done_t) - min(sub_t)
        ncell = float(sum(cells[k] for k in picks))
        worst = [{"model": str(pool[picks[i]]["model"]), "cells": cells[picks[i]], "latency_ms": round(1e3 * l, 1),
                  "queued_ms": round(1e3 * q, 1)} for l, i, q in sorted(slow, reverse=True)[:5]]
        return {"p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
                "slowest": worst,
                "mean_ms": 1e3 * float(np.mean(lat)), "solves_per_s": args.serve_requests / span,
                "cells_per_s": ncell / span, "batches": st["batches"], "max_batch": st["max_batch"],
                "peak_bytes": st["peak_bytes"]}

    # warm-up of both paths (every family's resident solver and the plain path)
    with Server(max_batch=args.serve_resident) as srv:
        for t in [srv.submit(pool[k]) for k in range(min(8, len(pool)))]:
            t.wait()
    with Server(max_batch=1) as srv:
        for t in [srv.submit(pool[k]) for k in range(min(4, len(pool)))]:
            t.wait()
    out = []
    for r in rates:
        served = run_arm(args.serve_resident, r, seed=11 + int(r))
        plain = run_arm(1, r, seed=11 + int(r))
        out.append({"rate_req_per_s": r, "served": served, "plain_one_at_a_time": plain,
                    "speedup_solves_per_s": served["solves_per_s"] / plain["solves_per_s"],
                    "p99_ratio_plain_over_served": plain["p99_ms"] / served["p99_ms"]})
    # FP32 served results against the FP64 path on a 1% sample (at least 2) of the pool
    errs = []
    with Server(max_batch=args.serve_resident) as srv:
        sample = list(range(0, len(pool), max(1, len(pool) // max(2, len(pool) // 100))))[:max(2, len(pool) // 100)]
        t32 = [srv.submit(pool[k]) for k in sample]
        t64 = [srv.submit(dict(pool[k], solverPrecision="float64")) for k in sample]
        for a, b in zip(t32, t64):
            v32, v64 = a.result()["values"], b.result()["values"]
            fin = np.isfinite(v64)
            errs.append(float(np.max(np.abs(v64[fin] - v32[fin])) / np.max(np.abs(v64[fin]))))
    return {"workload": "60% Riemann2 (64-1024), 25% Riemann3 (64-192, walls), 15% ReedsShepp2 (N x N x 60, "
                        "N 64-256), 1-4 seeds, FP32, Poisson arrivals",
            "requests_per_rate": args.serve_requests, "pool_payloads": len(pool), "resident_max": args.serve_resident,
            "size_note": f"{args.serve_requests} requests per rate (the config's 10,000 per rate would take hours "
                         f"for both arms at 6 rates)",
            "rates": out, "fp32_max_rel_err_vs_fp64": max(errs), "fp64_sample": len(errs),
            "input_generation_s": gen_s,
            "path": "serving.Server (hfm_server C ABI) from host arrays, H2D/D2H inside the latency"}


# ------------------------------------------------------------------------------- differentiation leg

def differentiation_leg(args):
    """TTI3 128^3 (10 m spacing, Thomsen vp/eps/delta and tilt), one source at the top-face centre,
    loss = sum over 64 top-face receivers of (T - T_obs)^2 with T_obs from vp with a +5% Gaussian
    blob; d loss / d vp through the torch.autograd.Function over the GPU adjoint, checked by
    central differences (step 1e-4 vp) at voxels drawn among those with a gradient."""
    import torch
    import hamiltonfastmarching_b200 as H
    from hamiltonfastmarching_b200 import workloads as W
    from hamiltonfastmarching_b200.autograd import arrival_times
    n, h = args.tti_side, 0.01
    p = W.tti3_case(n, h=h, seed=4)
    vp0 = p.pop("_vp")
    L = n * h
    obs = W.tti3_case(n, h=h, seed=4, blob=((0.5 * L, 0.5 * L, 0.35 * L), 0.12 * L, 0.05))
    vp_obs = obs.pop("_vp")
    rng = np.random.default_rng(7)
    rx = rng.integers(0, n, (64, 2))
    receivers = np.ravel_multi_index((rx[:, 0], rx[:, 1], np.zeros(64, int)), (n, n, n))
    q = dict(p, verbosity=0.0)
    H.run(q)  # warm-up
    t0 = time.perf_counter()
    out = H.run(q)
    fwd_s = time.perf_counter() - t0
    with torch.no_grad():
        t_obs = arrival_times(p, torch.from_numpy(vp0 / vp_obs)).reshape(-1)[receivers]

    def loss_of(vp):
        T = arrival_times(p, torch.from_numpy(vp0) / vp)
        return ((T.reshape(-1)[receivers] - t_obs) ** 2).sum()

    vp = torch.from_numpy(vp0.copy()).requires_grad_(True)
    t0 = time.perf_counter()
    loss = loss_of(vp)
    t1 = time.perf_counter()
    loss.backward()
    t2 = time.perf_counter()
    g = vp.grad.numpy().reshape(-1)
    cand = np.flatnonzero(np.abs(g) > 1e-2 * np.abs(g).max())
    cells = rng.choice(cand, min(args.tti_fd_voxels, len(cand)), replace=False) if len(cand) else []
    errs = []
    for cell in cells:
        d = 1e-4 * vp0.reshape(-1)[cell]
        vpp, vpm = vp0.copy().reshape(-1), vp0.copy().reshape(-1)
        vpp[cell] += d
        vpm[cell] -= d
        with torch.no_grad():
            fd = (loss_of(torch.from_numpy(vpp.reshape(vp0.shape))) -
                  loss_of(torch.from_numpy(vpm.reshape(vp0.shape)))).item() / (2 * d)
        errs.append(abs(g[cell] - fd) / max(abs(fd), 1e-12))
    res = {"workload": f"TTI3 {n}^3, h = 10 m, Thomsen vp in [1.5,4.5] km/s, eps/delta in [0,0.2], dip <= 30 deg; "
                       f"64 top-face receivers, T_obs from vp with a +5% Gaussian blob",
           "forward_solve_s": fwd_s, "gpu_solve_s": out["GPUSolveTime"], "n_accepted": out["nAccepted"],
           "grid_updates_per_s": out["nAccepted"] / fwd_s,
           "loss": float(loss.item()), "autograd_forward_s": t1 - t0, "autograd_backward_s": t2 - t1,
           "fd_voxels": len(errs), "fd_max_rel_err": max(errs) if errs else None,
           "fd_step": "1e-4 vp, central", "dtype": "f64"}
    # the reference's backward differentiation (FileHFM_TTI3, inspectSensitivity at the receivers
    # with the loss gradient 2 (T - T_obs) as weights) against the GPU's costSensitivity_0
    from oracle.refrun import have_reference, run_reference
    if not args.no_cpu_baseline and have_reference("TTI3"):
        T = out["values"].reshape(-1)[receivers]
        h_ = p["gridScale"]
        pts = np.column_stack([(rx + 0.5) * h_, np.full(64, 0.5 * h_)])
        wts = 2.0 * (T - t_obs.numpy())
        q = dict(p, inspectSensitivity=pts, inspectSensitivityWeights=wts, inspectSensitivityLengths=np.array([64.0]),
                 verbosity=0.0)
        t0 = time.perf_counter()
        gout = H.run(q)
        gpu_sens_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        ref = run_reference(q)
        ref_s = time.perf_counter() - t0
        if ref.get("retcode") == 0:
            a, b = ref["costSensitivity_0"], gout["costSensitivity_0"]
            res["reference_backward"] = {
                "costSensitivity_max_rel_diff": float(np.max(np.abs(a - b)) / np.max(np.abs(a))),
                "values_max_rel_diff": float(np.max(np.abs(ref["values"] - gout["values"])) / np.max(np.abs(ref["values"]))),
                "reference_wall_s": ref_s, "reference_fm_s": float(ref["FMCPUTime"]),
                "reference_stencil_s": float(ref["StencilCPUTime"]), "gpu_run_with_sensitivity_s": gpu_sens_s,
                "cores": 1, "kind": "reference"}
    return res


def geodesic_leg(args):
    """Geodesic backtracking throughput: Riemann2 1024^2 (anisotropy 8, smooth random orientation,
    two wall segments, one seed at the centre) with --geo-tips random tips, discrete solver, then the
    same tips with the ODE solver. GPU: the geodesic stage of one run (CUDA events around the
    warp-per-tip kernels and their copies, `GeodesicCPUTime`), and the whole run through the public
    call. CPU: the reference's FileHFM_Riemann2 on the same input with --geo-cpu-tips of the tips
    (its own `GeodesicCPUTime`, one core)."""
    import hamiltonfastmarching_b200 as H
    from hamiltonfastmarching_b200 import workloads as W
    n = args.geo_side
    p = W.riemann2_case(n, aniso=8.0, seed=11, seed_points=np.array([[0.5, 0.5]]))
    p["walls"] = np.zeros((n, n))
    p["walls"][n // 4, n // 8: 7 * n // 8] = 1.0
    p["walls"][3 * n // 4, 0: 5 * n // 8] = 1.0
    rng = np.random.default_rng(12)
    tips = rng.uniform(0.01, 0.99, (args.geo_tips, 2))
    q = dict(p, tips=tips, verbosity=0.0, exportValues=0.0)
    H.run(q)  # warm-up
    t0 = time.perf_counter()
    out = H.run(q)
    run_s = time.perf_counter() - t0
    gpu_s = float(out["GeodesicCPUTime"])
    npts = int(np.sum(out["geodesicLengths"]))
    res = {"workload": f"Riemann2 {n}^2, anisotropy 8, 2 wall segments, 1 seed; {len(tips)} random tips",
           "tips": len(tips), "points": npts, "mean_points_per_tip": npts / len(tips),
           "gpu_geodesic_s": gpu_s, "tips_per_s": len(tips) / gpu_s, "run_s": run_s,
           "gpu_solve_s": float(out["GPUSolveTime"]), "dtype": "f64"}
    from oracle.refrun import have_reference, run_reference
    if not args.no_cpu_baseline and have_reference("Riemann2") and args.geo_cpu_tips > 0:
        k = min(args.geo_cpu_tips, len(tips))
        ref = run_reference(dict(p, tips=tips[:k], verbosity=0.0, exportValues=0.0))
        if ref.get("retcode") == 0:
            cpu_s = float(ref["GeodesicCPUTime"])
            res["cpu_baseline"] = {"tips_per_s": k / cpu_s, "cores": 1, "kind": "reference",
                                   "sample": f"FileHFM_Riemann2 on the same input with the first {k} tips: "
                                             f"GeodesicCPUTime {cpu_s:.3f} s"}
            gk = int(np.sum(out["geodesicLengths"][:k]))
            rk = int(np.sum(ref["geodesicLengths"]))
            res["cpu_baseline"]["points_same_tips"] = {"gpu": gk, "reference": rk}
            res["speedup_tips_per_s_vs_1_core"] = res["tips_per_s"] / (k / cpu_s)
    # the same tips with the ODE solver (geodesicSolver = 'ODE')
    qo = dict(q, geodesicSolver="ODE")
    H.run(qo)
    out = H.run(qo)
    ode = {"gpu_geodesic_s": float(out["GeodesicCPUTime"]), "points": int(np.sum(out["geodesicLengths"]))}
    ode["tips_per_s"] = len(tips) / ode["gpu_geodesic_s"]
    if "cpu_baseline" in res:
        ref = run_reference(dict(p, tips=tips[:k], geodesicSolver="ODE", verbosity=0.0, exportValues=0.0))
        if ref.get("retcode") == 0:
            cpu_s = float(ref["GeodesicCPUTime"])
            ode["cpu_baseline"] = {"tips_per_s": k / cpu_s, "cores": 1, "kind": "reference",
                                   "sample": f"FileHFM_Riemann2, geodesicSolver ODE, first {k} tips: "
                                             f"GeodesicCPUTime {cpu_s:.3f} s"}
            ode["speedup_tips_per_s_vs_1_core"] = ode["tips_per_s"] / (k / cpu_s)
    res["ode"] = ode
    return res


# ------------------------------------------------------------------------------------- our arm

def summarize(line):
    """Headline figures of every leg in a few hundred bytes."""
    def r(x, d=3):
        return None if x is None else float(f"{x:.{d}g}")
    out = {"fp64_updates_per_s": r(line["value"]), "fp32_updates_per_s": r(line["fp32"]["value"]),
           "fp32_err": r(line["fp32"]["max_rel_err_vs_fp64"], 2), "roofline_frac": r(line["roofline"]["frac"], 3),
           "e2e_updates_per_s": r((line.get("e2e") or {}).get("value"))}
    b = line.get("batch")
    if b:
        out["batch"] = {"solves_per_s": r(b["batched"]["solves_per_s"]),
                        "plain_solves_per_s": r(b["plain_one_at_a_time"]["solves_per_s"]),
                        "speedup": r(b["speedup_solves_per_s"]), "speedup_tuned": r(b["speedup_autotuned_solves_per_s"]),
                        "fp32_err": r(b["fp32_max_rel_err_vs_fp64"], 2)}
    sv = line.get("serving")
    if sv:
        out["serving"] = {"fp32_err": r(sv["fp32_max_rel_err_vs_fp64"], 2), "rates": [
            {"rate": x["rate_req_per_s"], "solves_per_s": r(x["served"]["solves_per_s"]),
             "plain": r(x["plain_one_at_a_time"]["solves_per_s"]), "p50_ms": r(x["served"]["p50_ms"]),
             "p99_ms": r(x["served"]["p99_ms"]), "plain_p50_ms": r(x["plain_one_at_a_time"]["p50_ms"]),
             "plain_p99_ms": r(x["plain_one_at_a_time"]["p99_ms"])} for x in sv["rates"]]}
    d = line.get("differentiation")
    if d:
        out["differentiation"] = {"forward_s": r(d["forward_solve_s"]), "backward_s": r(d["autograd_backward_s"]),
                                  "fd_voxels": d["fd_voxels"], "fd_err": r(d["fd_max_rel_err"], 2),
                                  "vs_reference_sens": r((d.get("reference_backward") or {}).get("costSensitivity_max_rel_diff"), 2)}
    g = line.get("geodesics")
    if g:
        out["geodesics"] = {"tips_per_s": r(g["tips_per_s"]), "speedup_1core": r(g.get("speedup_tips_per_s_vs_1_core"))}
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    import hamiltonfastmarching_b200 as H
    from hamiltonfastmarching_b200 import _lib
    from hamiltonfastmarching_b200 import workloads as W

    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    from hamiltonfastmarching_b200.replicas import max_over_ranks

    L = _lib.load()
    n = args.side
    params = W.riemann3_case(n, seed=1 + rank)
    N = n ** 3
    metric_h = np.ascontiguousarray(params["metric"].reshape(N, 6))
    walls_h = np.ascontiguousarray((params["walls"] != 0).astype(np.uint8).reshape(N))
    # seeds -> row-major indices: floor((p - origin) / h), unique, increasing (as hfm_run places them)
    h = params["gridScale"]
    ijk = np.floor(params["seeds"] / h).astype(np.int64)
    seed_idx = np.unique(np.ravel_multi_index(ijk.T, (n, n, n))).astype(np.int64)
    seed_val = np.zeros(len(seed_idx), np.float64)

    metric_d = torch.from_numpy(metric_h).cuda()
    walls_d = torch.from_numpy(walls_h).cuda()
    values_d = torch.empty(N, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def make_args(precision):
        a = _lib.RiemannDeviceArgs()
        a.ndim = 3
        for i in range(3):
            a.dims[i] = n
            a.grid_scale[i] = params["gridScale"]
        a.dual = 0
        a.precision = precision
        a.sweeps_per_tile = 0
        a.metric = metric_d.data_ptr()
        a.walls = walls_d.data_ptr()
        a.nseeds = len(seed_idx)
        a.seed_index = seed_idx.ctypes.data
        a.seed_value = seed_val.ctypes.data
        a.values = values_d.data_ptr()
        a.stream = stream.cuda_stream
        return a

    err = ctypes.create_string_buffer(512)

    def solve(a, st):
        rc = L.hfm_solve_riemann_device(ctypes.byref(a), ctypes.byref(st), err, 512)
        if rc != 0:
            raise RuntimeError(f"solve failed ({rc}): {err.value.decode()}")

    results = {}
    values_by_prec = {}
    for prec in (64, 32):
        a = make_args(prec)
        st = _lib.SolveStats()
        for _ in range(args.warmup):
            solve(a, st)
        torch.cuda.synchronize()
        barrier()
        launches0 = ctypes.c_ulonglong()
        L.hfm_kernel_launches(ctypes.byref(launches0))
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        solve_ms, stencil_ms, stats = [], [], []
        with ClockSampler(local) as clk:
            torch.cuda.synchronize()
            start.record(stream)
            for _ in range(args.steps):
                solve(a, st)
                solve_ms.append(st.solve_ms)
                stencil_ms.append(st.stencil_ms)
                stats.append((st.n_accepted, st.rounds, st.tile_activations, st.local_solves))
            end.record(stream)
            torch.cuda.synchronize()
        barrier()
        launches1 = ctypes.c_ulonglong()
        L.hfm_kernel_launches(ctypes.byref(launches1))
        elapsed_ms = max_over_ranks(start.elapsed_time(end))
        values_by_prec[prec] = values_d.cpu().numpy().copy()
        nacc = stats[-1][0]
        results[prec] = {
            "elapsed_ms": elapsed_ms, "ms_per_step": elapsed_ms / args.steps,
            "value": world * nacc * args.steps / (elapsed_ms * 1e-3),
            "n_accepted": nacc, "solve_ms": statistics.mean(solve_ms), "stencil_ms": statistics.mean(stencil_ms),
            "rounds": stats[-1][1], "tile_activations": stats[-1][2], "local_solves": stats[-1][3],
            "launches": (launches1.value - launches0.value) // args.steps * args.steps,
            "clocks": clk.summary(),
        }

    # FP32 error against the FP64 path, finite cells
    v64, v32 = values_by_prec[64], values_by_prec[32]
    fin = np.isfinite(v64)
    fp32_err = float(np.max(np.abs(v64[fin] - v32[fin])) / np.max(np.abs(v64[fin])))

    # ---- end to end through the public API (host arrays in, host arrays out)
    e2e = None
    if args.e2e_steps > 0:
        hp = dict(params, verbosity=0.0)
        H.run(hp)  # warm
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            out = H.run(hp)
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        e2e = {"value": world * out["nAccepted"] * args.e2e_steps / e2e_s, "unit": "grid-updates/s",
               "h2d_bytes_per_step": int(metric_h.nbytes + walls_h.nbytes + params["seeds"].nbytes),
               "d2h_bytes_per_step": int(N * 8),
               "path": "HFMIO.run (hfm_run C ABI) from pageable numpy arrays, FP64"}

    r64 = results[64]
    peak, peak_kind = measured_peak_gbs()
    achieved = BYTES_PER_UPDATE[64] * r64["n_accepted"] / (r64["solve_ms"] * 1e-3) / 1e9
    traffic = profiled_traffic(f"riemann3_{n}_f64")
    roofline = {"bound": "hbm", "kernel": "fim_kernel<double,0,6,false>", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": traffic,
                "algorithmic_bytes_per_update": BYTES_PER_UPDATE[64],
                "note": "achieved = 57 B x nAccepted / solver-kernel CUDA-event time on the launching stream"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = reference_cpu_sample(n)
    batch = None
    if not args.no_batch:
        batch = batched_leg(args, rank, world)
    serving = None
    if not args.no_serve:
        serving = serving_leg(args, rank, world)
    diff = None
    if not args.no_diff and rank == 0:
        diff = differentiation_leg(args)
    geo = None
    if not args.no_geo and rank == 0:
        geo = geodesic_leg(args)

    if rank == 0:
        line = {
            "metric": "grid-updates/s", "value": r64["value"], "unit": "grid-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r64["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(n),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": r64["clocks"],
            "gpu_launches": r64["launches"],
            "n_accepted": r64["n_accepted"],
            "phases_ms": {"stencil_and_graph": r64["stencil_ms"], "solve": r64["solve_ms"]},
            "solver": {"rounds": r64["rounds"], "tile_activations": r64["tile_activations"],
                       "local_solves": r64["local_solves"]},
            "fp32": {"value": results[32]["value"], "ms_per_step": results[32]["ms_per_step"],
                     "solve_ms": results[32]["solve_ms"], "max_rel_err_vs_fp64": fp32_err,
                     "clocks": results[32]["clocks"]},
            "batch": batch,
            "serving": serving,
            "differentiation": diff,
            "geodesics": geo,
        }
        # the compact digest (batch and serving speed-ups, p50/p99, FP32 errors) goes right after the
        # headline keys, before the long per-leg data, so that a record keeping only the beginning
        # of the line still has it
        digest = summarize(line)
        ordered = {}
        for k, v in line.items():
            ordered[k] = v
            if k == "gpu_launches":
                ordered["summary"] = digest
        print(json.dumps(ordered), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------------------ reference arm

def run_reference_arm(args):
    """The reference's own CPU implementation on the benchmarked workload: one step is one full
    FileHFM_Riemann3 solve (the reference's executable, compiled from its sources, single-threaded)
    of the 192^3 instance, from its input file to its output file. Steps run concurrently, one
    process per host core (a pool over the steps); value = steps x nAccepted / wall time of the
    timed steps. Warm-up steps run the same way before the timed region."""
    import concurrent.futures as cf
    rank, world, _ = rank_env()
    if rank != 0:
        return
    from oracle.refrun import have_reference, ref_executable, read_output, write_input
    from hamiltonfastmarching_b200 import workloads as W
    n = args.side
    if not have_reference("Riemann3"):
        print(json.dumps({"impl": "reference", "unavailable": "reference FileHFM_Riemann3 not built (make -C oracle ref)"}))
        return
    cores = os.cpu_count() or 1
    p = W.riemann3_case(n, seed=1)
    p["exportValues"] = 0.0
    tmp = tempfile.mkdtemp(prefix="hfmrefbench_")
    write_input(p, os.path.join(tmp, "input"))
    del p
    exe = ref_executable("Riemann3")
    counter = iter(range(1 << 30))

    def one_solve(_):
        out = os.path.join(tmp, f"out{next(counter)}")
        subprocess.run([exe, os.path.join(tmp, "input"), out], stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL, check=True)
        r = read_output(out)
        for ext in ("_Format.txt", "_Data.dat"):
            os.unlink(out + ext)
        return r

    def run_steps(k):
        with cf.ThreadPoolExecutor(max_workers=max(1, min(cores, k))) as ex:
            return list(ex.map(one_solve, range(k)))

    if args.warmup > 0:
        run_steps(args.warmup)
    t0 = time.perf_counter()
    outs = run_steps(args.steps)
    el = time.perf_counter() - t0
    nacc = outs[-1]["nAccepted"]
    value = nacc * args.steps / el
    waves = -(-args.steps // cores)
    cpu_s = statistics.mean(o["FMCPUTime"] + o["StencilCPUTime"] for o in outs)
    line = {"impl": "reference", "metric": "grid-updates/s", "value": value, "unit": "grid-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(n),
            "cpu_baseline": {"value": value, "unit": "grid-updates/s", "cores": min(cores, args.steps), "kind": "reference",
                             "sample": f"{args.steps} full solves of the {n}^3 instance by FileHFM_Riemann3 (reference "
                                       f"code, one thread each), {min(cores, args.steps)} at a time on {cores} host "
                                       f"cores ({waves} wave(s)); {int(nacc)} reached cells per solve; mean "
                                       f"FMCPUTime + StencilCPUTime {cpu_s:.1f} s per solve"},
            "e2e": {"value": value, "unit": "grid-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    import shutil
    shutil.rmtree(tmp, ignore_errors=True)


def main(argv=None):
    args = parse_args(argv)
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
