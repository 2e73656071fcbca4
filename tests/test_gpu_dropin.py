"""The C++ drop-in layer (include/qkxTM_b200.hpp): a driver written like the
reference's bin/test_applyTM.cpp / bin/test_invert.cpp, compiled with g++
against libqkx_b200.so and run on the GPU, checked against the oracle."""
import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_cpp_dropin_driver(qkx, oracle, tmp_path):
    exe = str(tmp_path / "test_dropin")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "test_dropin.cpp"),
           "-L", os.path.join(ROOT, "qkxtm_mpi_b200"), "-lqkx_b200",
           "-L", os.path.join(ROOT, "oracle"), "-l:liboracle.so",
           f"-Wl,-rpath,{os.path.join(ROOT, 'qkxtm_mpi_b200')}", f"-Wl,-rpath,{os.path.join(ROOT, 'oracle')}",
           "-o", exe]
    subprocess.run(cmd, check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")
