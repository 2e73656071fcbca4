"""CPU tests of the C-ABI boundary: the library builds, loads, and exports every
entry point declared in include/*.h; argument checking happens before any
CUDA call.  No compute is run here."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT, gpu_available


def _header_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(qkx_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


@pytest.fixture(scope="module")
def built_lib():
    from qkxtm_mpi_b200 import build
    if not os.path.exists(build.LIB):
        build.build()
    return build.LIB


def test_header_declares_the_package_symbols():
    import qkxtm_mpi_b200 as Q
    assert _header_functions() == set(Q.SYMBOLS)


def test_library_exports_every_declared_symbol(built_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", built_lib], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = _header_functions() - exported
    assert not missing, missing
    # nothing else leaks out of the library under a qkx_ prefix
    extra = {s for s in exported if s.startswith("qkx_")} - _header_functions()
    assert not extra, extra


def test_library_loads_and_reports_version(built_lib):
    import qkxtm_mpi_b200 as Q
    assert "sm_100a" in Q.version()
    assert Q.lib().qkx_last_error() is not None


def test_parameter_checks_need_no_device(built_lib):
    import qkxtm_mpi_b200 as Q
    L = Q.lib()
    ctx = C.c_void_p()
    bad = [
        Q.LatticeInfo(L=(3, 4, 4, 4)),           # odd L[0]: the even-odd layout needs it even
        Q.LatticeInfo(L=(4, 4, 4, 1)),           # extent below 2
        Q.LatticeInfo(L=(4, 4, 4, 4), twistSign=2),
        Q.LatticeInfo(L=(4, 4, 4, 4), boundaryT=0),
    ]
    for info in bad:
        p = info.to_c()
        rc = L.qkx_create(C.byref(p), 0, C.byref(ctx))
        assert rc == Q.ERR_INVALID
        assert L.qkx_last_error().decode().startswith("invalid argument")
        assert not ctx.value
    assert L.qkx_create(None, 0, C.byref(ctx)) == Q.ERR_INVALID


def test_null_context_is_rejected(built_lib):
    import qkxtm_mpi_b200 as Q
    L = Q.lib()
    assert L.qkx_apply(None, 0, None, None) == Q.ERR_INVALID
    assert L.qkx_load_gauge(None, None, 0) == Q.ERR_INVALID
    assert L.qkx_spinor_bytes(None) == 0
    L.qkx_destroy(None)


def test_create_without_gpu_fails_cleanly(built_lib):
    if gpu_available():
        pytest.skip("a GPU is present")
    import qkxtm_mpi_b200 as Q
    with pytest.raises(Q.QkxError) as e:
        Q.Lattice(Q.LatticeInfo(L=(4, 4, 4, 4)))
    assert e.value.code == Q.ERR_CUDA


def test_cpp_dropin_header_compiles():
    """include/qkxTM_b200.hpp (the reference-named C++ layer) is valid C++17."""
    src = os.path.join(ROOT, "tests", "cpp", "test_dropin.cpp")
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), src], check=True)


# C structs of include/qkx_b200.h and their ctypes mirrors in the Python binding
_STRUCTS = {
    "qkx_params": "Params",
    "qkx_solve_info": "SolveInfo",
    "qkx_solver_params": "SolverParams",
    "qkx_batch_job": "BatchJob",
    "qkx_lime_info": "LimeInfo",
    "qkx_ptc_params": "PtcParams",
    "qkx_ptc_train_params": "PtcTrainParams",
    "qkx_ptc_train_info": "PtcTrainInfo",
}


def test_struct_layouts_match_the_header(tmp_path):
    """Every ctypes structure of the binding has the size and field offsets of its C struct,
    as a C compiler lays it out from the header (a mismatch would shift the fields that
    follow, e.g. the status and message of a batch job after its solve info)."""
    import qkxtm_mpi_b200 as Q
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "qkx_b200.h"', "int main(void) {"]
    for cname, pyname in _STRUCTS.items():
        cls = getattr(Q, pyname)
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layouts.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layouts"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            name, key, val = line.split()
            got[(name, key)] = int(val)
    for cname, pyname in _STRUCTS.items():
        cls = getattr(Q, pyname)
        assert got[(cname, "size")] == C.sizeof(cls), (cname, got[(cname, "size")], C.sizeof(cls))
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)
