"""The allocation-free dot product (qkx_reCdotXdagY_noalloc), called through the
C ABI.  It exists for callers that cannot allocate device memory (their
device memory is owned by another allocator or a fixed budget, or their path
must not enter the allocator), so it cannot use a context's buffers; it keeps
its scratch in a fixed array inside the library.  Its result must equal the
context-based reCdotXdagY on the same device fields, on consecutive calls.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative, as the FP64 BLAS tests


def _noalloc(qkx, x, y, sites, stream):
    out = C.c_double(float("nan"))
    qkx.check(qkx.lib().qkx_reCdotXdagY_noalloc(x.ptr, y.ptr, sites, C.byref(out), stream))
    return out.value


def test_noalloc_dot_matches_context_dot_on_consecutive_calls(qkx, oracle):
    # two calls in a row on different lattices, so the second (smaller) call
    # would expose any partial sums left behind by the first
    for L, seed in (((8, 8, 8, 16), 1), ((4, 4, 4, 8), 2)):
        with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
            x = lat.field(oracle.spinor_gaussian(L, seed))
            y = lat.field(oracle.spinor_gaussian(L, seed + 10))
            ref = lat.reCdotXdagY(x, y)
            got = _noalloc(qkx, x, y, lat.V, lat.stream())
            assert abs(got - ref) <= TOL * abs(ref)
            again = _noalloc(qkx, x, x, lat.V, None)  # default stream, |x|^2
            assert abs(again - lat.norm2(x)) <= TOL * abs(again)
            x.close()
            y.close()


def test_noalloc_rejects_sizes_above_its_limit(qkx, oracle):
    L = (4, 4, 4, 4)
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        x = lat.field(oracle.spinor_gaussian(L, 3))
        out = C.c_double()
        rc = qkx.lib().qkx_reCdotXdagY_noalloc(x.ptr, x.ptr, qkx.NOALLOC_MAX_SITES + 1, C.byref(out), None)
        assert rc == qkx.ERR_INVALID
        assert "limit" in qkx.lib().qkx_last_error().decode()
        x.close()


def test_noalloc_rejects_unaligned_and_host_pointers_before_launch(qkx, oracle):
    # both cases are turned into QKX_ERR_INVALID on the host, before any kernel runs
    import numpy as np
    L = (4, 4, 4, 4)
    with qkx.Lattice(qkx.LatticeInfo(L=L)) as lat:
        x = lat.field(oracle.spinor_gaussian(L, 4))
        out = C.c_double()
        rc = qkx.lib().qkx_reCdotXdagY_noalloc(x.ptr + 8, x.ptr, 16, C.byref(out), None)
        assert rc == qkx.ERR_INVALID
        assert "aligned" in qkx.lib().qkx_last_error().decode()
        host = np.zeros(12 * 2 * lat.V, dtype=np.float64)
        rc = qkx.lib().qkx_reCdotXdagY_noalloc(x.ptr, host.ctypes.data_as(C.c_void_p), lat.V, C.byref(out), None)
        assert rc == qkx.ERR_INVALID
        assert "device memory" in qkx.lib().qkx_last_error().decode()
        # the library still works after the rejections
        assert abs(_noalloc(qkx, x, x, lat.V, None) - lat.norm2(x)) <= TOL * lat.norm2(x)
        x.close()
