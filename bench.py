#!/usr/bin/env python
"""Benchmark of the twisted-mass Dslash / CG hot path on B200.

Workload (the 12-source multi-RHS solve): 32^3 x 64 lattice, synthetic links
U = exp(i 0.3 H) (seeded), antiperiodic time boundary, kappa = 0.1615,
mu = 0.0015, the 12 spin-colour point sources at the origin, every source
solved to a true residual ||b - M x|| / ||b|| <= 1e-10 recomputed in FP64.

A step is one solve of all 12 sources (time to solution).  `value` is the
device time of a step with inputs resident in HBM (even-odd mixed-precision
CG, all sources in one batch, CUDA-graph iterations); `e2e` is the same step
through the host-buffer C ABI (qkx_load_gauge + qkx_invert from page-locked
host memory, solutions read back).  The plain FP64 CG of the reference's
algorithm on the same GPU is timed beside it (`plain_fp64_s`).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank solves its own 12 sources (point sources on
time slice 2*rank): weak scaling, no data-path collective; `value` is the
max over ranks of the per-step device time.
`--impl reference` times the reference's own CPU code (compiled from its
sources, oracle/_ref) on the host cores instead.

Other workloads (one JSON line each, same --steps/--warmup rules, 1 GPU):
  --workload propagator  the smeared-source propagator of bin/test_invert_prop.cpp
                         (APE 20 x 0.5, Gaussian 50 x 4.0 at source and sink, 12
                         point sources, mixed solver to 1e-10) at 32^3x64
  --workload uneven      four lattices 16^3x32 .. 32^3x64 with their own links
                         (eps ~ U[0.2, 0.35]) and masses {0.0015, 0.004, 0.01},
                         12 solves of 4 Gaussian sources, run concurrently
  --workload ptc         the learned preconditioner at 32^3x64: 64 training solves,
                         --ptc-steps Adam steps, then the 12 point sources in one batch by
                         flexible CG on the even-odd system, preconditioned by the network
  --workload contract    the 10 meson and 4 nucleon two-point functions with 33
                         momenta (Q^2 <= 4) from a 32^3x64 propagator in HBM
  --workload dslash      the Dslash alone: the 12-RHS even-odd hop in FP16 and FP32
                         (autotuned tile) and the FP64 full-lattice M, in GB/s
--lattice X,Y,Z,T replaces 32^3x64 in the non-default workloads (small cases for
profiling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L = (32, 32, 32, 64)
KAPPA, MU, EPS, SEED, NSRC, TOL = 0.1615, 0.0015, 0.3, 1234, 12, 1e-10
WORKLOAD = (f"twisted-mass CG, {L[0]}^3x{L[3]}, {NSRC} spin-colour point sources, "
            f"kappa={KAPPA}, mu={MU}, eps={EPS}, antiperiodic t, true residual <= {TOL:g}")
METRIC = "CG time-to-solution at 1e-10, 12 point sources, 32^3x64 (mu=0.0015)"
FALLBACK_HBM_GBS = 6650.0


def env_rank():
    from qkxtm_mpi_b200.dist import env_rank as er
    return er()


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples of one GPU during a region (200 ms period)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        ids = [v.strip() for v in vis.split(",")] if vis else None
        self.gpu = ids[local_rank] if ids and local_rank < len(ids) else str(local_rank)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                rows.append((float(f[0]), float(f[1]), f[4:8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, fl in rows for i, v in enumerate(fl) if v == "Active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def point_sources(np, t_src: int, Ls=None):
    Ls = Ls or L
    V = Ls[0] * Ls[1] * Ls[2] * Ls[3]
    site = Ls[0] * Ls[1] * Ls[2] * t_src
    out = []
    for s in range(4):
        for c in range(3):
            b = np.zeros((V, 4, 3, 2))
            b[site, s, c, 0] = 1.0
            out.append(b)
    return out


# --------------------------------------------------------------------------- ours
def run_ours(args):
    import numpy as np
    import torch

    import qkxtm_mpi_b200 as Q
    from qkxtm_mpi_b200 import dist as D

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        D.init("nccl", local)
    prec = {"half": Q.PREC_HALF, "single": Q.PREC_SINGLE, "double": Q.PREC_DOUBLE}[args.precision]
    V = L[0] * L[1] * L[2] * L[3]

    lat = Q.Lattice(Q.LatticeInfo(L=L, kappa=KAPPA, mu=MU, twistSign=1, boundaryT=-1, tol=TOL,
                                  maxIter=5000), device=local)
    lat.generate_gauge(EPS, SEED, Q.LINKS_APPLY_BC)
    t_src = D.source_timeslice(rank, L[3])
    srcs = point_sources(np, t_src)
    bd = [lat.field(b) for b in srcs]
    xd = [lat.field() for _ in srcs]
    stream = torch.cuda.ExternalStream(lat.stream())

    def solve():
        info = lat.invert_dev(bd, xd, method=Q.SOLVER_CG_EO_MIXED, precision=prec, tol=TOL,
                              maxIter=5000)
        if not (info.converged and info.true_residual <= TOL):
            raise RuntimeError(f"solve did not converge: {info.as_dict()}")
        return info

    barrier = D.barrier

    # autotune the inner hop for this lattice and batch (cached in the context), or use
    # the tile given on the command line (so that a profiler run launches the same kernel)
    if args.tile:
        tile = list(args.tile) + [0] * (3 - len(args.tile))
        lat.set_tile(prec, NSRC, tile)
    else:
        lat.tune(prec, NSRC)
        tile = min(lat.tune_table(prec, NSRC), key=lambda e: e["ms_per_hop"])["tile"]
    for _ in range(args.warmup):
        solve()
    lat.sync()

    # ---- timed region: inputs resident in HBM; each solve is one graph launch (the iteration
    # loop runs on the device) plus the set-up and final kernels
    barrier()
    torch.cuda.synchronize()
    k0 = lat.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    infos = []
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            infos.append(solve())
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    launches = lat.kernel_launches() - k0
    ms = D.max_over_ranks(e0.elapsed_time(e1))
    step_s = ms / 1e3 / args.steps

    # ---- the dominant kernel, timed: the same solves with CUDA events recorded around every
    # sloppy hop on the library's stream (the solver then runs its host-driven loop, one graph
    # per iteration, because event records cannot sit inside the device loop's conditional
    # nodes; the kernels and their inputs are the same)
    lat.profile_reset()
    lat.profile(True)
    for _ in range(max(1, min(args.steps, 3))):
        solve()
    lat.sync()
    hop_n, hop_ms, hop_bytes = lat.profile_read()
    lat.profile(False)

    # ---- end to end through the host-buffer C ABI
    Uh = Q.pinned_array((V, 4, 3, 3, 2))
    Uh[...] = lat.download_gauge()
    bh = [Q.pinned_array((V, 4, 3, 2)) for _ in srcs]
    for h, b in zip(bh, srcs):
        h[...] = b
    xh = [Q.pinned_array((V, 4, 3, 2)) for _ in srcs]

    def e2e_step():
        lat.load_gauge(Uh, Q.LINKS_AS_GIVEN)
        _, info = lat.invert(bh, method=Q.SOLVER_CG_EO_MIXED, precision=prec, tol=TOL, maxIter=5000,
                             out=xh)
        return info

    e2e_step()
    n_e2e = max(1, min(args.steps, 3))
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = D.max_over_ranks((time.perf_counter() - t0) / n_e2e)
    h2d = Uh.nbytes + sum(b.nbytes for b in bh)
    d2h = sum(x.nbytes for x in xh)

    # ---- the plain FP64 method (the reference's algorithm) on the same GPU
    plain = None
    if not args.no_plain:
        torch.cuda.synchronize()
        pinfo = lat.invert_dev(bd, xd, method=Q.SOLVER_CG_FP64, tol=TOL, maxIter=5000)
        plain = {"seconds": pinfo.seconds, "iterations": pinfo.iterations,
                 "true_residual": pinfo.true_residual}

    # ---- CPU baseline (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import cpu_baseline as CB
        iters = plain["iterations"] if plain else None
        cb = CB.run(L, KAPPA, MU, EPS, SEED, n_sources=NSRC, n_iter=1, iters_full=iters,
                    links=np.array(Uh))
        cpu = {"value": cb["value"], "unit": "s", "cores": cb["cores"], "kind": cb["kind"],
               "sample": cb["sample"]}

    D.finish()
    if rank != 0:
        return

    peak, peak_src = measured_peak_hbm()
    avg_launch_ms = hop_ms / max(hop_n, 1)
    bytes_per_launch = hop_bytes / max(hop_n, 1)
    achieved = bytes_per_launch / (avg_launch_ms * 1e-3) / 1e9 if hop_n else None
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "hop_traffic.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            tj = json.load(f)
        key = f"{args.precision}_kind{tile[2]}"
        if key in tj:
            # ncu DRAM bytes per output site per RHS of the captured launch, scaled to this launch
            traffic = tj[key]["dram_bytes_per_site_rhs"] * (V // 2) * NSRC
    it = max(i.iterations for i in infos)
    line = {
        "metric": METRIC,
        "value": step_s,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_s * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"half": "f16 storage / f32 accumulate / f64 reliable updates, solution and residual",
                  "single": "f32 storage / f32 accumulate / f64 reliable updates, solution and residual",
                  "double": "f64"}[args.precision],
        "data": "synthetic (seeded exp(i eps H) links, point sources)",
        "config": {"workload": WORKLOAD, "lattice": "x".join(map(str, L)), "sources_per_gpu": NSRC,
                   "solver": ("even-odd CG, all sources in one batch; the iteration loop is one CUDA graph "
                              "launch (conditional WHILE nodes, decisions on the device)"),
                   "storage": {"half": "fp16 spinors", "single": "fp32 spinors",
                               "double": "fp64 spinors"}[args.precision] + " + " + hop_links(args.precision, tile),
                   "accumulate": "fp32 inner, fp64 reliable updates / solution / residual checks",
                   "l2": "inputs larger than L2 (links alone 201 MB fp16, spinor batches > 600 MB)",
                   "parallelism": f"replicas x{world} (independent sources per GPU)"},
        "iterations": it,
        "reliable_updates": max(i.reliable_updates for i in infos),
        "true_residual_max": max(i.true_residual for i in infos),
        # device time per solve by phase (medians over the timed solves)
        "phases_s": {k: round(float(np.median([getattr(i, a) for i in infos])), 5) for k, a in (
            ("setup", "seconds_setup"), ("reliable_updates", "seconds_reliable"), ("final", "seconds_final"),
            ("solve", "seconds"))},
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": {
            "kernel": (f"{hop_kernel_name(args.precision, tile)}<{args.precision} spinors, "
                       f"{hop_links(args.precision, tile)}, "
                       f"{NSRC}-RHS batch, {tile[0]} RHS/thread, {tile[1]} threads/block, kind {tile[2]}>"),
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "peak_source": peak_src,
            "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None,
            "traffic": traffic,
            "launches": hop_n,
            "timed": "CUDA events around each sloppy hop in profiled solves of the same workload",
            "avg_launch_ms": avg_launch_ms,
            "algorithmic_bytes_per_launch": bytes_per_launch,
        },
        "clocks": clk.summary(),
    }
    if plain:
        line["plain_fp64_s"] = plain["seconds"]
        line["plain_fp64_iterations"] = plain["iterations"]
        line["speedup_vs_plain_fp64"] = plain["seconds"] / step_s
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- reference
def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return
    import numpy as np
    from oracle import cpu_baseline as CB
    from oracle import oracle as O

    O.build(ref=True)
    links = O.apply_bc(L, O.gauge_random(L, EPS, SEED), -1)
    path = CB.write_links(links)  # once for every step
    del links
    # iterations of the reference's CG recurrence to a true residual of 1e-10, from a small lattice
    # (solved once, cached by cpu_baseline)
    vals, last = [], None
    try:
        for i in range(args.warmup + args.steps):
            last = CB.run(L, KAPPA, MU, EPS, SEED, n_sources=NSRC, n_iter=1, iters_full=None, links_path=path)
            if i >= args.warmup:
                vals.append(last["value"])
    finally:
        os.unlink(path)
    value = statistics.median(vals)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": value * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded exp(i eps H) links, point sources)",
        "config": {"workload": WORKLOAD, "lattice": "x".join(map(str, L)), "sources_per_gpu": NSRC,
                   "solver": "reference CG::operator() on M^+M (lib/solvers.cpp), FP64, host cores"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": last["cores"], "kind": last["kind"],
                         "sample": last["sample"]},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    del np
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- other workloads
def _common(args, metric, value, unit, higher, workload, extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": higher, "scaling": "weak", "vs_baseline": None,
            "data": "synthetic (seeded links and sources)", "config": {"workload": workload}}
    line.update(extra)
    print(json.dumps(line), flush=True)


def _events(Q, lat):
    import torch
    stream = torch.cuda.ExternalStream(lat.stream())
    return stream, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _roofline(kernel, launches, ms, nbytes, traffic=None):
    peak, src = measured_peak_hbm()
    avg = ms / max(launches, 1)
    per = nbytes / max(launches, 1)
    ach = per / (avg * 1e-3) / 1e9 if launches else None
    return {"kernel": kernel, "bound": "hbm", "achieved": ach, "peak": peak, "peak_source": src, "unit": "GB/s",
            "frac": ach / peak if ach else None, "traffic": traffic, "launches": launches, "avg_launch_ms": avg,
            "algorithmic_bytes_per_launch": per}


def hop_links(precision, tile):
    """The link format a sloppy-hop tile reads."""
    if precision in ("half", "fp16") and tile[2] == 9:
        return "18-real fp32 links"
    if precision in ("half", "fp16") and tile[2] in (10, 11):
        return "18-real fp16 links"
    return {"half": "12-real fp16 links", "fp16": "12-real fp16 links", "single": "12-real fp32 links",
            "double": "18-real fp64 links"}[precision]


def hop_link_bytes(precision, tile):
    """Bytes of one link in the format a sloppy-hop tile reads."""
    return {"12-real fp16 links": 24.0, "18-real fp16 links": 36.0, "12-real fp32 links": 48.0,
            "18-real fp32 links": 72.0, "18-real fp64 links": 144.0}[hop_links(precision, tile)]


def hop_kernel_name(precision, tile):
    """The sloppy hop kernel a tile (rhs_per_thread, threads_per_block, kind) launches."""
    if 1 <= tile[2] <= 3:
        return "hop_pair_pf_kernel"
    if tile[2] == 10:
        return "hop_pair_hm_kernel"
    if tile[2] >= 8:
        return "hop_pair_hp_kernel"
    if tile[2] >= 5:
        return "hop_pair_as_kernel"
    if precision in ("half", "fp16") and tile[0] % 2 == 0:
        return "hop_pair_kernel"
    return "hop_mrhs_kernel"


def run_dslash(args):
    import numpy as np
    import torch
    import qkxtm_mpi_b200 as Q
    torch.cuda.set_device(0)
    Lw = args.lattice
    lat = Q.Lattice(Q.LatticeInfo(L=Lw, kappa=KAPPA, mu=MU, boundaryT=-1))
    lat.generate_gauge(EPS, SEED, Q.LINKS_APPLY_BC)
    Vh = lat.V // 2
    hops = {}
    with ClockSampler(0) as clk:
        for name, prec, S in (("fp16", Q.PREC_HALF, 52.0), ("fp32", Q.PREC_SINGLE, 96.0)):
            # CUDA events around 3 repetitions of the solver's four-hop iteration per tile, best tile
            nr, nt, ms = lat.tune(prec, NSRC)
            table = lat.tune_table(prec, NSRC)
            best = min(table, key=lambda e: e["ms_per_hop"])["tile"]
            # one output parity, averaged over the four hops: input spinor and 8 links shared by the
            # batch, the output spinor (hops 1-3), the xpay operand (hops 2 and 4), and the FP32 CG
            # residual read and written by the fourth hop's epilogue
            G = hop_link_bytes({"fp16": "half", "fp32": "single"}[name], best)
            nbytes = Vh * NSRC * ((9.0 * S + 2.0 * 96.0) / 4.0 + 8.0 * G / NSRC)
            hops[name] = {"tile": best, "ms_per_hop": ms, "gbs": nbytes / (ms * 1e-3) / 1e9,
                          "algorithmic_bytes_per_hop": nbytes,
                          "tiles_ms_per_hop": {",".join(map(str, e["tile"])): round(e["ms_per_hop"], 4)
                                               for e in table}}
        a = lat.field(np.random.default_rng(1).standard_normal((lat.V, 4, 3, 2)))
        b = lat.field()
        for _ in range(args.warmup):
            lat.apply_dev("tm", a, b)
        lat.sync()
        lat.profile_reset()
        lat.profile(True)
        for _ in range(args.steps):
            lat.apply_dev("tm", a, b)
        lat.sync()
        n, ms, by = lat.profile_read()
        lat.profile(False)
    a.close()
    b.close()
    fp64 = {"launches": n, "ms": ms / max(n, 1), "gbs": by / (ms * 1e-3) / 1e9,
            "gflops": 1416.0 * lat.V * n / (ms * 1e-3) / 1e9}
    peak, src = measured_peak_hbm()
    lat_s = "x".join(map(str, Lw))
    _common(args, f"Dslash HBM GB/s: even-odd hop, {NSRC} RHS, FP16 spinors and 12-real links, {lat_s}",
            hops["fp16"]["gbs"], "GB/s", True,
            f"{hop_kernel_name('half', hops['fp16']['tile'])} on one parity of {lat_s} for a batch of {NSRC} "
            f"right-hand sides (autotuned tile {hops['fp16']['tile']}), "
            f"kappa={KAPPA}, mu={MU}; FP64 full-lattice M beside it",
            {"dtype": "f16 storage / f32 arithmetic", "fp16": hops["fp16"], "fp32": hops["fp32"], "fp64_tm": fp64,
             "roofline": {"kernel": hop_kernel_name("half", hops["fp16"]["tile"]) + "<fp16>", "bound": "hbm",
                          "achieved": hops["fp16"]["gbs"],
                          "peak": peak, "peak_source": src, "unit": "GB/s", "frac": hops["fp16"]["gbs"] / peak,
                          "traffic": None, "algorithmic_bytes_per_launch": hops["fp16"]["algorithmic_bytes_per_hop"],
                          "avg_launch_ms": hops["fp16"]["ms_per_hop"]},
             "gpu_launches": lat.kernel_launches(), "clocks": clk.summary()})


def run_propagator(args):
    import numpy as np
    import torch
    import qkxtm_mpi_b200 as Q
    torch.cuda.set_device(0)
    NS, AL, NA, AA = 50, 4.0, 20, 0.5
    L = args.lattice
    lat = Q.Lattice(Q.LatticeInfo(L=L, kappa=KAPPA, mu=MU, boundaryT=-1))
    lat.generate_gauge(EPS, SEED, Q.LINKS_AS_GIVEN)
    U = Q.pinned_array((lat.V, 4, 3, 3, 2))
    U[...] = lat.download_gauge()
    lat.APE_smearing(U, NA, AA, download=False)  # smearing links from the links without the boundary sign
    lat.load_gauge(U, Q.LINKS_APPLY_BC)
    lat.tune(Q.PREC_HALF, NSRC)
    nbytes = lat.V * 2304
    dprop = Q.lib().qkx_device_alloc(lat.ctx, nbytes)
    stream, e0, e1 = _events(Q, lat)

    def step():
        info = lat.propagator_dev(dprop, (0, 0, 0, 0), NS, AL, tol=TOL)
        if not info.converged:
            raise RuntimeError("propagator solve did not converge")
        return info

    for _ in range(args.warmup):
        step()
    lat.sync()
    k0 = lat.kernel_launches()
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            info = step()
        e1.record(stream)
        torch.cuda.synchronize()
    launches = lat.kernel_launches() - k0
    step_s = e0.elapsed_time(e1) / 1e3 / args.steps
    # the Gaussian smearing kernel alone: 12 fields, 10 full-lattice steps
    fs = [lat.field(np.random.default_rng(k).standard_normal((lat.V, 4, 3, 2))) for k in range(NSRC)]
    gs = [lat.field() for _ in range(NSRC)]
    lat.Gaussian_smearing_dev(fs, gs, 1, AL)
    lat.sync()
    lat.profile_reset()
    lat.profile(True)
    lat.Gaussian_smearing_dev(fs, gs, 10, AL)
    lat.sync()
    n, ms, by = lat.profile_read()
    lat.profile(False)
    for f in fs + gs:
        f.close()
    # end to end: host links in, host propagator out
    out = Q.pinned_array((lat.V, 4, 4, 3, 3, 2))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    n_e2e = max(1, min(args.steps, 2))
    for _ in range(n_e2e):
        lat.load_gauge(U, Q.LINKS_APPLY_BC)
        lat.APE_smearing(U, NA, AA, download=False)
        lat.propagator((0, 0, 0, 0), NS, AL, tol=TOL, out=out)
    e2e_s = (time.perf_counter() - t0) / n_e2e
    Q.lib().qkx_device_free(lat.ctx, dprop)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import cpu_baseline as CB
        cpu = CB.propagator_sample(L, KAPPA, MU, EPS, SEED, NS, AL)
    _common(args, "smeared-source propagator time (12 point sources, 32^3x64)", step_s, "s", False,
            f"APE {NA}x{AA}, Gaussian {NS}x{AL} at source and sink, 12 point sources, mixed solver to {TOL:g}, "
            f"32^3x64, kappa={KAPPA}, mu={MU}",
            {"ms_per_step": step_s * 1e3, "dtype": "f64 smearing / f16-f32-f64 solver",
             "iterations": info.iterations, "true_residual_max": info.true_residual,
             "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 2 * U.nbytes,
                     "d2h_bytes_per_step": out.nbytes},
             "gpu_launches": launches,
             "roofline": _roofline("k_gauss_step (12 fields, FP64, 18-real links)", n, ms, by),
             "clocks": clk.summary(), **({"cpu_baseline": cpu} if cpu else {})})


def run_uneven(args):
    import numpy as np
    import torch
    import qkxtm_mpi_b200 as Q
    torch.cuda.set_device(0)
    lattices = [(16, 16, 16, 32), (20, 20, 20, 40), (24, 24, 24, 48), (32, 32, 32, 64)]
    masses = [0.0015, 0.004, 0.01]
    rng = np.random.default_rng(SEED)
    lats, jobs, fields = [], [], []
    for i, Li in enumerate(lattices):
        eps = float(rng.uniform(0.2, 0.35))
        lat = Q.Lattice(Q.LatticeInfo(L=Li, kappa=KAPPA, mu=MU, boundaryT=-1))
        lat.generate_gauge(eps, SEED + i, Q.LINKS_APPLY_BC)
        lat.tune(Q.PREC_HALF, 4)
        lats.append((lat, eps))
        for j in range(3):
            bs = [lat.field(np.random.default_rng(1000 * i + 10 * j + k).standard_normal((lat.V, 4, 3, 2)))
                  for k in range(4)]
            xs = [lat.field() for _ in range(4)]
            fields += bs + xs
            jobs.append((lat, bs, xs, [masses[(j + k) % 3] for k in range(4)]))
    for _ in range(args.warmup):
        Q.invert_batch(jobs, tol=TOL)
    lats_k0 = sum(l.kernel_launches() for l, _ in lats)
    lat_all, steps_s = [], []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = Q.invert_batch(jobs, tol=TOL)
            torch.cuda.synchronize()
            steps_s.append(time.perf_counter() - t0)
            lat_all += [r["latency"] for r in res]
            if not all(r["info"]["converged"] for r in res):
                raise RuntimeError("a batched solve did not converge")
    launches = sum(l.kernel_launches() for l, _ in lats) - lats_k0
    step_s = statistics.median(steps_s)
    nrhs = 4 * len(jobs)
    p50, p99 = float(np.percentile(lat_all, 50)), float(np.percentile(lat_all, 99))
    # end to end: sources from pinned host memory, solutions back
    hb = [Q.pinned_array((l.V, 4, 3, 2)) for (l, bs, xs, m) in jobs for _ in bs]
    for i, h in enumerate(hb):
        h[...] = np.random.default_rng(7000 + i).standard_normal(h.shape)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    k = 0
    for (l, bs, xs, m) in jobs:
        for b in bs:
            Q.check(Q.lib().qkx_spinor_upload(l.ctx, hb[k].ctypes.data, b.ptr))
            k += 1
    Q.invert_batch(jobs, tol=TOL)
    k = 0
    for (l, bs, xs, m) in jobs:
        for x in xs:
            Q.check(Q.lib().qkx_spinor_download(l.ctx, x.ptr, hb[k].ctypes.data))
            k += 1
    e2e_s = time.perf_counter() - t0
    nb = sum(h.nbytes for h in hb)
    for f in fields:
        f.close()
    _common(args, "batched uneven solves: right-hand sides per second (4 lattices, 12 solves x 4 RHS)",
            nrhs / step_s, "rhs/s", True,
            "16^3x32, 20^3x40, 24^3x48, 32^3x64 with eps ~ U[0.2,0.35]; 3 solves x 4 Gaussian RHS each, "
            "mu in {0.0015, 0.004, 0.01}; even-odd mixed CG to 1e-10; lattices concurrent on one GPU",
            {"ms_per_step": step_s * 1e3, "dtype": "f16 storage / f32 accumulate / f64 reliable",
             "latency_p50_s": p50, "latency_p99_s": p99, "batch_seconds": step_s,
             "eps": [e for _, e in lats],
             "e2e": {"value": nrhs / e2e_s, "unit": "rhs/s", "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb},
             "gpu_launches": launches, "clocks": clk.summary()})


# the learned preconditioner's network: six parallel-transport layers with 16 hidden channels, in
# colour-vector channels (4 spin channels in and out; a channel is a colour 3-vector, so the layers
# commute with gauge transformations).  Four layers (--ptc-widths 4,16,16,16,4) do not shorten the
# solve on this configuration; six halve its iterations.
PTC_WIDTHS = (4, 16, 16, 16, 16, 16, 4)


def run_ptc(args):
    import numpy as np
    import torch
    import qkxtm_mpi_b200 as Q
    torch.cuda.set_device(0)
    L = args.lattice
    lat = Q.Lattice(Q.LatticeInfo(L=L, kappa=KAPPA, mu=MU, boundaryT=-1))
    lat.generate_gauge(EPS, SEED, Q.LINKS_APPLY_BC)
    lat.tune(Q.PREC_HALF, NSRC)
    widths = args.ptc_widths or PTC_WIDTHS
    net = Q.Ptc(lat, widths, seed=3, init_scale=0.05, tensor_cores=True)
    train = net.train(n_solves=64, steps=args.ptc_steps, lr=3e-3, solve_tol=1e-6, seed=9)
    srcs = point_sources(np, 0, L)
    bd = [lat.field(b) for b in srcs]
    xd = [lat.field() for _ in srcs]

    def solve(pre):
        return lat.invert_dev(bd, xd, method=Q.SOLVER_GCR_PTC, tol=TOL, preconditioner=pre)

    for _ in range(args.warmup):
        solve(net)
    stream, e0, e1 = _events(Q, lat)
    k0 = lat.kernel_launches()
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            info = solve(net)
        e1.record(stream)
        torch.cuda.synchronize()
    launches = lat.kernel_launches() - k0
    step_s = e0.elapsed_time(e1) / 1e3 / args.steps
    plain_gcr = solve(None)
    mixed = lat.invert_dev(bd, xd, method=Q.SOLVER_CG_EO_MIXED, tol=TOL)
    fp64 = lat.invert_dev(bd, xd, method=Q.SOLVER_CG_FP64, tol=TOL, maxIter=5000)
    # end to end from host buffers
    bh = [Q.pinned_array((lat.V, 4, 3, 2)) for _ in srcs]
    for h, b in zip(bh, srcs):
        h[...] = b
    xh = [Q.pinned_array((lat.V, 4, 3, 2)) for _ in srcs]
    t0 = time.perf_counter()
    lat.invert(bh, method=Q.SOLVER_GCR_PTC, tol=TOL, out=xh, preconditioner=net)
    e2e_s = time.perf_counter() - t0
    for f in bd + xd:
        f.close()
    net.close()
    _common(args, "learned-preconditioned CG time-to-solution at 1e-10, 12 point sources, 32^3x64", step_s, "s",
            False, f"PTC {len(widths) - 1} layers {'-'.join(map(str, widths))} colour-vector channels, BF16 "
                   f"weights and activations, tcgen05 16->16 layers; 64 training solves, {args.ptc_steps} Adam steps; "
                   f"all 12 sources in one batch on the even-odd Schur system: flexible CG on its normal "
                   f"equations in FP32, preconditioned by K K^+ (K the network on the even sites), FP64 defect "
                   f"correction; "
                   f"kappa={KAPPA}, mu={MU}",
            {"ms_per_step": step_s * 1e3, "dtype": "bf16 network / f32 CG / f64 residual",
             "iterations": info.iterations, "fallbacks": info.fallbacks, "true_residual_max": info.true_residual,
             "training": train,
             "compare": {"same_solver_no_preconditioner": {"seconds": plain_gcr.seconds,
                                                           "iterations": plain_gcr.iterations,
                                                           "fallbacks": plain_gcr.fallbacks},
                         "mixed_cg": {"seconds": mixed.seconds, "iterations": mixed.iterations},
                         "plain_fp64_cg": {"seconds": fp64.seconds, "iterations": fp64.iterations}},
             "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": sum(b.nbytes for b in bh),
                     "d2h_bytes_per_step": sum(x.nbytes for x in xh)},
             "gpu_launches": launches, "clocks": clk.summary()})


def run_contract(args):
    import numpy as np
    import torch
    import qkxtm_mpi_b200 as Q
    torch.cuda.set_device(0)
    L = args.lattice
    Qsq = 4
    lat = Q.Lattice(Q.LatticeInfo(L=L))
    V = lat.V
    host = Q.pinned_array((V, 4, 4, 3, 3, 2))
    host[...] = np.random.default_rng(SEED).standard_normal(host.shape)
    nbytes = V * 2304
    d = Q.lib().qkx_device_alloc(lat.ctx, nbytes)
    Q.check(Q.lib().qkx_memcpy_h2d(lat.ctx, d, host.ctypes.data, nbytes))

    def step():
        lat.meson_2pt(d, range(10), Qsq, (0, 0, 0, 0), device=True)
        for op in range(4):
            lat.baryon_2pt(d, d, op, Qsq, (0, 0, 0, 0), device=True)

    for _ in range(args.warmup):
        step()
    k0 = lat.kernel_launches()
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
        torch.cuda.synchronize()
        step_s = (time.perf_counter() - t0) / args.steps
    launches = lat.kernel_launches() - k0
    t0 = time.perf_counter()
    lat.meson_2pt(host, range(10), Qsq)
    for op in range(4):
        lat.baryon_2pt(host, host, op, Qsq)
    e2e_s = time.perf_counter() - t0
    Q.lib().qkx_device_free(lat.ctx, d)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import cpu_baseline as CB
        cpu = CB.contract_sample(L, Qsq)
    nmom = len(Q.momenta(Qsq))
    _common(args, "two-point functions per propagator: 10 mesons + 4 nucleon operators, 33 momenta, 32^3x64",
            step_s, "s", False, f"Meson::contract x10 + Baryon::contract x4 + Fourier to {nmom} momenta "
                                f"(Q^2 <= {Qsq}) from a 32^3x64 propagator in HBM",
            {"ms_per_step": step_s * 1e3, "dtype": "f64",
             "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 9 * host.nbytes,
                     "d2h_bytes_per_step": 8 * L[3] * nmom * (10 + 4 * 16) * 2},
             "gpu_launches": launches, "clocks": clk.summary(), **({"cpu_baseline": cpu} if cpu else {})})


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["half", "single", "double"], default="half")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--workload", choices=["cg", "propagator", "uneven", "ptc", "contract", "dslash"],
                    default="cg")
    ap.add_argument("--ptc-steps", type=int, default=2000)
    ap.add_argument("--ptc-widths", type=lambda v: tuple(int(x) for x in v.split(",")), default=None,
                    help="channel widths of the learned preconditioner's network (default 4,16,16,16,16,16,4)")
    ap.add_argument("--lattice", type=lambda v: tuple(int(x) for x in v.split(",")), default=L,
                    help="X,Y,Z,T for the non-default workloads")
    ap.add_argument("--tile", type=lambda v: tuple(int(x) for x in v.split(",")), default=None,
                    help="RHS_PER_THREAD,THREADS_PER_BLOCK,KIND of the sloppy hop instead of the autotuner's")
    args = ap.parse_args()
    if args.warmup < 3:
        print("note: --warmup below 3 raised to 3", file=sys.stderr)
        args.warmup = 3
    if args.impl == "reference":
        if args.workload != "cg":
            print(json.dumps({"impl": "reference", "unavailable": "the reference arm is defined for the default "
                              "workload; the other workloads carry their own cpu_baseline"}), flush=True)
            return
        run_reference(args)
    elif args.workload == "cg":
        run_ours(args)
    else:
        {"propagator": run_propagator, "uneven": run_uneven, "ptc": run_ptc, "contract": run_contract,
         "dslash": run_dslash}[args.workload](args)


if __name__ == "__main__":
    main()
