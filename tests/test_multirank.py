"""The benchmark's multi-GPU plumbing on CPU: two gloo ranks, each with its
own sources, timings reduced with the max over ranks (no GPU needed)."""
import os
import socket
import subprocess
import sys

from conftest import ROOT

WORKER = r"""
import os, sys, json
sys.path.insert(0, os.environ["QKX_ROOT"])
from qkxtm_mpi_b200 import dist as D
rank, world, local = D.env_rank()
D.init("gloo")
t = D.source_timeslice(rank, 64)
D.barrier()
mx = D.max_over_ranks(1.5 + rank)
D.barrier()
D.finish()
print(json.dumps({"rank": rank, "world": world, "t": t, "max": mx}))
"""


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_shard_sources_and_reduce_max(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    port = _port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), QKX_ROOT=ROOT)
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    import json
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(o["rank"] for o in outs) == [0, 1]
    assert all(o["max"] == 2.5 for o in outs)           # max over ranks reaches every rank
    assert len({o["t"] for o in outs}) == 2              # each rank has its own sources


def test_single_process_needs_no_group():
    from qkxtm_mpi_b200 import dist as D
    assert D.max_over_ranks(3.0) == 3.0
    assert D.source_timeslice(0, 64) == 0 and D.source_timeslice(33, 64) == 2


SOLVE_WORKER = r"""
import os, sys, json, time
sys.path.insert(0, os.environ["QKX_ROOT"])
import numpy as np
from qkxtm_mpi_b200 import dist as D
from oracle import oracle as O
rank, world, local = D.env_rank()
D.init("gloo", timeout_s=60)
L, kappa, mu = (4, 4, 4, 8), 0.16, 0.01
U = O.apply_bc(L, O.gauge_random(L, 0.3, 7), -1)        # every rank holds the same links (replicas)
t = D.source_timeslice(rank, L[3])
D.barrier()
t0 = time.perf_counter()
worst = 0.0
for s in range(2):                                      # this rank's own point sources
    b = O.spinor_point(L, (0, 0, 0, t), s, 0)
    x, _, _ = O.cg(L, U, O.apply("tm_dag", L, U, b, kappa, mu), kappa, mu, tol=1e-12, maxIter=2000)
    r = b - O.apply("tm", L, U, x, kappa, mu)
    worst = max(worst, float(np.linalg.norm(r) / np.linalg.norm(b)))
el = time.perf_counter() - t0
D.barrier()
mx = D.max_over_ranks(el)
D.finish()
print(json.dumps({"rank": rank, "t": t, "worst": worst, "elapsed": el, "max": mx}))
"""

FAIL_WORKER = r"""
import os, sys, json, time
sys.path.insert(0, os.environ["QKX_ROOT"])
from qkxtm_mpi_b200 import dist as D
rank, world, local = D.env_rank()
D.init("gloo", timeout_s=20)
D.barrier()
if rank == 1:
    raise SystemExit(3)                                 # a rank that leaves between steps
t0 = time.perf_counter()
try:
    D.max_over_ranks(1.0)
    print(json.dumps({"rank": rank, "detected": False}))
except Exception as e:                                  # the peer's loss ends the collective
    print(json.dumps({"rank": rank, "detected": True, "after_s": time.perf_counter() - t0}))
"""


def _launch(tmp_path, source, world=2, timeout=240):
    script = tmp_path / "worker.py"
    script.write_text(source)
    port = _port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), QKX_ROOT=ROOT)
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    res = []
    for p in procs:
        out, err = p.communicate(timeout=timeout)
        res.append((p.returncode, out, err))
    return res


def test_two_ranks_solve_their_own_sources(tmp_path):
    """The bench's replica scheme run as solves: each gloo rank solves its own point sources (the
    oracle's CG standing in for the GPU solver on CPU ranks), the ranks' times meet in one max."""
    import json
    res = _launch(tmp_path, SOLVE_WORKER)
    outs = []
    for rc, out, err in res:
        assert rc == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(o["rank"] for o in outs) == [0, 1]
    assert len({o["t"] for o in outs}) == 2
    assert all(o["worst"] <= 1e-10 for o in outs), outs
    assert all(o["max"] == max(p["elapsed"] for p in outs) for o in outs)


def test_a_rank_that_leaves_ends_the_others_collective(tmp_path):
    """Failure detection on the host: a rank exits between steps, and the next collective of the
    one that stays ends with an error instead of waiting for good."""
    import json
    res = _launch(tmp_path, FAIL_WORKER, timeout=180)
    rc0, out0, err0 = res[0]
    assert res[1][0] == 3
    assert rc0 == 0, err0[-2000:]
    o = json.loads(out0.strip().splitlines()[-1])
    assert o["detected"] is True and o["after_s"] < 60, o
