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
