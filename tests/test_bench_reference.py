"""CPU test of bench.py's reference arm: it runs the reference's own CG, compiled
from its sources, on the host cores and prints one JSON line with the keys the
measurement contract asks for; on a rank other than 0 it exits without work."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def _run(env_extra, timeout):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)


def test_reference_arm_prints_the_contract_line():
    from oracle import oracle as O
    O.build(ref=True)
    if not O.ref_available():
        pytest.skip("the reference sources are not present to build the reference CG")
    r = _run({}, 600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "dtype", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["unit"] == "s" and line["higher_is_better"] is False
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work():
    r = _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"}, 120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
