"""Timed CPU baseline of the hot path: the reference's own CG (oracle/_ref,
compiled from the reference sources) or, where that build is absent, the
oracle's C restatement, run on the host cores.

TEST/BASELINE INFRASTRUCTURE ONLY: used by the CPU-baseline leg and the
reference arm of bench.py, never by the product path.

The reference is single-threaded (its only parallelism is MPI ranks), so the
host cores are used the way the reference would use them for a multi-source
job: one independent single-rank process per source.  A bounded sample --
`n_iter` CG iterations in each of P concurrent processes on the full lattice --
gives the time per CG iteration under full-socket load; the projection to the
whole job is  ceil(n_sources / P) * iterations_to_converge * t_iteration.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

from oracle import oracle as O


def _worker(args):
    kind, L, kappa, mu, links_path, spin, colour, n_iter = args
    L = tuple(L)
    V = O.volume(L)
    U = np.fromfile(links_path, dtype=np.float64).reshape(V, 4, 3, 3, 2)
    b = O.spinor_point(L, (0, 0, 0, 0), spin, colour)
    x = np.zeros_like(b)
    if kind == "reference":
        lib = O.ref()
        lib.ref_cg_timed.restype = C.c_double
        lib.ref_cg_timed.argtypes = [O._ip, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int,
                                     O._dp, O._dp, O._dp]
        return lib.ref_cg_timed(O._L(L), kappa, mu, 1, 1e-30, n_iter, O._ptr(U), O._ptr(b), O._ptr(x))
    t0 = time.perf_counter()
    O.cg(L, U, b, kappa, mu, 1, tol=1e-30, maxIter=n_iter)
    return time.perf_counter() - t0


_ITERS_CACHE: dict = {}


def iterations_to_converge(L, kappa, mu, eps, seed, tol=1e-10) -> tuple[int, float]:
    """Iterations the reference's CG recurrence (lib/solvers.cpp:16-81) needs on
    a lattice small enough to solve quickly, same parameters, point source, to
    reach a TRUE residual ||b - M x|| / ||b|| <= tol.

    The reference stops on the normal-equation residual r2 <= tol^2 |M^+ b|^2,
    which leaves the true residual somewhat above tol; the stop is tightened
    (and the solve repeated from zero) until the true residual meets tol, as the
    GPU's plain FP64 CG does.  Returns (iterations, true residual reached); the
    result is cached per parameter set for the life of the process."""
    key = (tuple(L), kappa, mu, eps, seed, tol)
    if key not in _ITERS_CACHE:
        _ITERS_CACHE[key] = _iterations_to_converge(L, kappa, mu, eps, seed, tol)
    return _ITERS_CACHE[key]


def _iterations_to_converge(L, kappa, mu, eps, seed, tol):
    U = O.apply_bc(L, O.gauge_random(L, eps, seed), -1)
    b = O.spinor_point(L, (0, 0, 0, 0), 0, 0)
    Mdb = O.apply("tm_dag", L, U, b, kappa, mu, 1)
    nb = float(np.linalg.norm(b))
    stop = tol
    for _ in range(20):
        x, k, _ = O.cg(L, U, Mdb, kappa, mu, 1, tol=stop, maxIter=5000)
        true = float(np.linalg.norm(b - O.apply("tm", L, U, x, kappa, mu, 1)) / nb)
        if true <= tol:
            return k, true
        stop *= 0.5 * tol / true
    return k, true


def write_links(links: np.ndarray) -> str:
    """The links as a raw FP64 file for the worker processes (in /dev/shm when it has
    room); the caller removes it."""
    import shutil
    tmpdir = tempfile.gettempdir()
    if os.path.isdir("/dev/shm") and shutil.disk_usage("/dev/shm").free > 2 * links.nbytes:
        tmpdir = "/dev/shm"
    fd, path = tempfile.mkstemp(prefix="qkx_links_", suffix=".f64", dir=tmpdir)
    os.close(fd)
    links.astype(np.float64).tofile(path)
    return path


def run(L, kappa, mu, eps, seed, n_sources=12, n_iter=1, procs=None, iters_full=None,
        links: np.ndarray | None = None, timeout: float = 900.0, links_path: str | None = None) -> dict:
    """Time the CPU hot path and project it to solving n_sources point sources.
    links_path: the links already written by write_links (kept), else they are
    written for this call and removed after it.

    Returns {"value": seconds for the whole job, "per_iter_s", "cores", "kind",
    "sample", "iters_full"}."""
    O.build(ref=True)
    kind = "reference" if O.ref_available() else "port"
    ncpu = os.cpu_count() or 1
    P = max(1, min(n_sources, ncpu if procs is None else procs))
    own = links_path is None
    if own:
        if links is None:
            links = O.apply_bc(L, O.gauge_random(L, eps, seed), -1)
        path = write_links(links)
    else:
        path = links_path
    try:
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        env = dict(os.environ, PYTHONPATH=root + os.pathsep + os.environ.get("PYTHONPATH", ""))
        t0 = time.perf_counter()
        procs_ = []
        for i in range(P):
            job = [kind, list(L), kappa, mu, path, (i // 3) % 4, i % 3, n_iter]
            procs_.append(subprocess.Popen([sys.executable, "-m", "oracle.cpu_baseline", json.dumps(job)],
                                           cwd=root, env=env, stdout=subprocess.PIPE, text=True))
        times = []
        deadline = time.time() + timeout
        for p in procs_:
            try:
                out, _ = p.communicate(timeout=max(1.0, deadline - time.time()))
            except subprocess.TimeoutExpired:
                for q in procs_:
                    q.kill()
                raise RuntimeError("CPU baseline worker timed out")
            if p.returncode != 0:
                raise RuntimeError(f"CPU baseline worker failed (rc={p.returncode})")
            times.append(float(out.strip().splitlines()[-1]))
        wall = time.perf_counter() - t0
    finally:
        if own:
            os.unlink(path)
    per_iter = float(np.median(times)) / n_iter
    if iters_full is None:
        small = (8, 8, 8, 16)
        iters_full, true = iterations_to_converge(small, kappa, mu, eps, seed)
        src = (f"iterations of the reference's CG recurrence on {small[0]}^3x{small[3]}, its stop tightened "
               f"until the true residual ||b-Mx||/||b|| = {true:.2e} <= 1e-10")
    else:
        src = ("iterations of the reference's CG recurrence at full size (the GPU's FP64 replica), its stop "
               "tightened until the true residual ||b-Mx||/||b|| <= 1e-10")
    value = math.ceil(n_sources / P) * iters_full * per_iter
    sample = (f"{P} concurrent single-rank {kind} CG processes x {n_iter} iteration(s) on "
              f"{L[0]}x{L[1]}x{L[2]}x{L[3]} (median {per_iter:.2f} s/iteration under full load, "
              f"wall {wall:.1f} s); projected to {n_sources} sources x {iters_full} iterations "
              f"({src})")
    return {"value": value, "per_iter_s": per_iter, "cores": P, "kind": kind, "sample": sample,
            "iters_full": iters_full}


def propagator_sample(L, kappa, mu, eps, seed, nsmear, alpha, n_sources=12, small=(16, 16, 16, 32)) -> dict:
    """The reference's smeared-source propagator loop (bin/test_invert_prop.cpp:83-97)
    on the host: per source two Gaussian smearings of nsmear steps and one CG
    solve.  The smearing is timed with the reference's Vector::Gaussian_smearing
    (2 steps of one vector on `small`) and scaled by volume; the solves come from
    run() (concurrent single-rank processes, as for the CG baseline)."""
    O.build(ref=True)
    kind = "reference" if O.ref_available() else "port"
    U = O.gauge_random(small, eps, seed)
    psi = O.spinor_gaussian(small, seed + 1)
    smear = O.ref_gaussian_smear if kind == "reference" else O.gaussian_smear
    t0 = time.perf_counter()
    smear(small, U, psi, 2, alpha)
    t_step = (time.perf_counter() - t0) / 2 * (O.volume(L) / O.volume(small))
    cg = run(L, kappa, mu, eps, seed, n_sources=n_sources, n_iter=1)
    P = cg["cores"]
    smear_total = math.ceil(n_sources / P) * 2 * nsmear * t_step
    value = smear_total + cg["value"]
    sample = (f"{kind} Gaussian_smearing, 2 steps of one vector on {'x'.join(map(str, small))} scaled by volume "
              f"({t_step:.2f} s/step at full size) x 2 x {nsmear} steps per source; solves: {cg['sample']}")
    return {"value": value, "unit": "s", "cores": P, "kind": kind, "sample": sample}


def contract_sample(L, Q_sq, small=(8, 8, 8, 16)) -> dict:
    """The reference's Meson::contract x10 and Baryon::contract x4 with their
    Fourier transforms, timed on `small` (one process) and scaled by volume:
    both the site contractions and the transform are linear in V."""
    O.build(ref=True)
    kind = "reference" if O.ref_available() else "port"
    V = O.volume(small)
    rng = np.random.default_rng(1)
    p = rng.standard_normal((V, 4, 4, 3, 3, 2))
    meson = O.ref_meson_2pt if kind == "reference" else O.meson_2pt
    baryon = O.ref_baryon_2pt if kind == "reference" else O.baryon_2pt
    t0 = time.perf_counter()
    for op in range(10):
        meson(small, p, op, Q_sq)
    for op in range(4):
        baryon(small, p, p, op, Q_sq)
    t = time.perf_counter() - t0
    value = t * O.volume(L) / V
    sample = (f"{kind} contractions (10 mesons + 4 nucleon operators, Q^2 <= {Q_sq}) on "
              f"{'x'.join(map(str, small))} in {t:.2f} s, scaled by volume to {'x'.join(map(str, L))}")
    return {"value": value, "unit": "s", "cores": 1, "kind": kind, "sample": sample}


if __name__ == "__main__":
    # worker process: time n_iter CG iterations and print the seconds
    print(_worker(json.loads(sys.argv[1])), flush=True)
