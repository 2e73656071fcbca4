"""qkxtm_mpi_b200 -- the twisted-mass Dslash / CG hot path of qkxTM_MPI on B200.

This module is a thin ctypes layer over the C ABI in ``include/qkx_b200.h``
(``libqkx_b200.so``, built in-tree by ``qkxtm_mpi_b200.build``).  It mirrors the
reference's hot-path interface by name:

* ``LatticeInfo``            -- struct LatticeInfo (include/qkxTM.h:156-204)
* ``Lattice.tm / tmDag / tmDagtm / Wilson / tm_xx / tm_xxDagTm_xx / *_chiral``
                             -- qkxTM::Vector members (lib/lattice_util.cpp:1148-2071)
* ``Lattice.cg``             -- CG::operator() (lib/solvers.cpp:16-81)
* ``Lattice.reCdotXdagY / X_eq_X_p_aY / X_eq_aX_p_Y / norm2``
                             -- lib/blas_qkxTM.cpp, Vector::norm2
* ``Lattice.invert``         -- the solve sequence tmDag + CG of bin/test_invert.cpp,
                                with the B200 solvers (plain FP64 or even-odd mixed precision)
* ``Lattice.calculatePlaquette / APE_smearing / Gaussian_smearing / absorbVector``
                             -- Gauge / Vector / Propagator members (lib/lattice_util.cpp:923-1145, 2073)
* ``Lattice.propagator``     -- the smeared-source propagator loop of bin/test_invert_prop.cpp

Fields are numpy float64 arrays in the reference's host layouts: spinor
``[V, 4, 3, 2]`` (Vector::M) and gauge ``[V, 4, 3, 3, 2]`` (Gauge::M).

There is no CPU fallback: importing works without a GPU, but every call that
computes goes through the CUDA library and raises ``QkxError`` if it is
missing or fails.
"""
from __future__ import annotations

import ctypes as C
import weakref
import os
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqkx_b200.so")

OK = 0
ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_NOGAUGE, ERR_NOT_CONVERGED, ERR_NAN, ERR_UNSUPPORTED = (
    -1, -2, -3, -4, -5, -6, -7)

LINKS_AS_GIVEN, LINKS_APPLY_BC = 0, 1
NOALLOC_MAX_SITES = 11184810  # QKX_NOALLOC_MAX_SITES
LINKS_OPERATOR, LINKS_SMEARING = 0, 1
SOLVER_CG_FP64, SOLVER_CG_EO_MIXED, SOLVER_GCR_PTC = 0, 1, 2
PREC_DOUBLE, PREC_SINGLE, PREC_HALF = 0, 1, 2

# operator ids of enum qkx_op
OPS = {
    "dslash": 0, "dslash_dag": 1, "tm": 2, "tm_dag": 3, "tm_dagtm": 4, "wilson": 5,
    "tm_xx_ee": 6, "tm_xx_oo": 7, "tm_xx_dagtm_xx_ee": 8, "tm_xx_dagtm_xx_oo": 9,
    "dslash_chiral": 10, "tm_chiral": 11, "tm_xx_chiral_ee": 12, "tm_xx_chiral_oo": 13,
    "tm_xx_dagtm_xx_chiral_ee": 14, "tm_xx_dagtm_xx_chiral_oo": 15, "gamma5": 16,
    "gamma5_chiral": 17, "twist": 18, "twist_inv": 19, "twist_dag": 20, "twist_dag_inv": 21,
    "twist_inv_chiral": 22, "dslash_xx_eo": 23, "dslash_xx_oe": 24,
    "rotate_chiral_to_ukqcd": 25, "dslash_xx_chiral_eo": 26, "dslash_xx_chiral_oe": 27,
    "tm_dag_chiral": 28, "tm_dagtm_chiral": 29,
}

# exported symbols of include/qkx_b200.h (checked by the CPU tests)
SYMBOLS = [
    "qkx_version", "qkx_last_error", "qkx_create", "qkx_destroy", "qkx_set_params",
    "qkx_get_params", "qkx_sync", "qkx_stream", "qkx_spinor_bytes", "qkx_volume",
    "qkx_load_gauge", "qkx_gauge_generate", "qkx_download_gauge", "qkx_gauge_compressible",
    "qkx_apply", "qkx_apply_dev", "qkx_spinor_upload", "qkx_spinor_download",
    "qkx_reCdotXdagY", "qkx_X_eq_X_p_aY", "qkx_X_eq_aX_p_Y", "qkx_norm2", "qkx_reCdotXdagY_noalloc",
    "qkx_cg", "qkx_cg_dev", "qkx_invert", "qkx_invert_dev",
    "qkx_host_alloc", "qkx_host_free", "qkx_device_alloc", "qkx_device_free",
    "qkx_memcpy_h2d", "qkx_memcpy_d2h",
    "qkx_profile_enable", "qkx_profile_read", "qkx_profile_reset", "qkx_kernel_launches", "qkx_tune",
    "qkx_set_tile", "qkx_tune_table", "qkx_sloppy_normal",
    "qkx_plaquette", "qkx_plaquette_loaded", "qkx_project_su3", "qkx_ape_smear", "qkx_load_smearing_gauge",
    "qkx_gaussian_smear", "qkx_gaussian_smear_dev", "qkx_propagator_absorb", "qkx_propagator",
    "qkx_propagator_dev", "qkx_ptc_create", "qkx_ptc_destroy", "qkx_ptc_num_weights", "qkx_ptc_get_weights",
    "qkx_ptc_set_weights", "qkx_ptc_apply", "qkx_ptc_loss_grad", "qkx_ptc_train",
    "qkx_read_gauge_lime", "qkx_write_gauge_lime", "qkx_momenta", "qkx_meson_2pt", "qkx_meson_2pt_dev",
    "qkx_baryon_2pt", "qkx_baryon_2pt_dev", "qkx_delta_2pt", "qkx_delta_2pt_dev", "qkx_nucleon_2pt",
    "qkx_nucleon_2pt_dev", "qkx_invert_batch",
]


class QkxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"qkx error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [("L", C.c_int * 4), ("kappa", C.c_double), ("mu", C.c_double),
                ("twistSign", C.c_int), ("boundaryT", C.c_int), ("tol", C.c_double),
                ("maxIter", C.c_int), ("reliableDelta", C.c_double)]


class SolverParams(C.Structure):
    _fields_ = [("method", C.c_int), ("sloppy_precision", C.c_int), ("tol", C.c_double),
                ("maxIter", C.c_int), ("reliable_delta", C.c_double), ("use_graphs", C.c_int),
                ("mu", C.POINTER(C.c_double)), ("preconditioner", C.c_void_p)]


PTC_MAX_LAYERS = 8


class PtcParams(C.Structure):
    _fields_ = [("nlayers", C.c_int), ("channels", C.c_int * (PTC_MAX_LAYERS + 1)), ("seed", C.c_ulonglong),
                ("init_scale", C.c_double), ("tensor_cores", C.c_int)]


class PtcTrainParams(C.Structure):
    _fields_ = [("n_solves", C.c_int), ("steps", C.c_int), ("lr", C.c_double), ("solve_tol", C.c_double),
                ("seed", C.c_ulonglong)]


class PtcTrainInfo(C.Structure):
    _fields_ = [("loss_initial", C.c_double), ("loss_final", C.c_double), ("seconds_data", C.c_double),
                ("seconds_train", C.c_double), ("steps", C.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class LimeInfo(C.Structure):
    _fields_ = [("precision", C.c_int), ("L", C.c_int * 4), ("data_offset", C.c_longlong),
                ("data_bytes", C.c_longlong), ("records", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("reliable_updates", C.c_int), ("converged", C.c_int),
                ("restarts", C.c_int), ("true_residual", C.c_double),
                ("normal_residual", C.c_double), ("seconds", C.c_double), ("fallbacks", C.c_int),
                ("seconds_setup", C.c_double), ("seconds_reliable", C.c_double), ("seconds_final", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchJob(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("nrhs", C.c_int), ("b_dev", C.POINTER(C.c_void_p)),
                ("x_dev", C.POINTER(C.c_void_p)), ("mu", C.POINTER(C.c_double)), ("status", C.c_int),
                ("latency", C.c_double), ("info", SolveInfo), ("message", C.c_char * 160)]


_lib = None
_vp, _dp = C.c_void_p, C.POINTER(C.c_double)


def lib() -> C.CDLL:
    """Load libqkx_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise QkxError(ERR_UNSUPPORTED,
                           f"{LIB_PATH} is missing: run `python -m qkxtm_mpi_b200.build`")
        L = C.CDLL(LIB_PATH)
        L.qkx_version.restype = C.c_char_p
        L.qkx_last_error.restype = C.c_char_p
        L.qkx_create.argtypes = [C.POINTER(Params), C.c_int, C.POINTER(_vp)]
        L.qkx_destroy.argtypes = [_vp]
        L.qkx_destroy.restype = None
        L.qkx_set_params.argtypes = [_vp, C.POINTER(Params)]
        L.qkx_get_params.argtypes = [_vp, C.POINTER(Params)]
        L.qkx_sync.argtypes = [_vp]
        L.qkx_stream.argtypes = [_vp]
        L.qkx_stream.restype = _vp
        L.qkx_spinor_bytes.argtypes = [_vp]
        L.qkx_spinor_bytes.restype = C.c_size_t
        L.qkx_volume.argtypes = [_vp]
        L.qkx_volume.restype = C.c_size_t
        L.qkx_load_gauge.argtypes = [_vp, _vp, C.c_int]
        L.qkx_gauge_generate.argtypes = [_vp, C.c_double, C.c_ulonglong, C.c_int]
        L.qkx_download_gauge.argtypes = [_vp, _vp]
        L.qkx_gauge_compressible.argtypes = [_vp]
        L.qkx_apply.argtypes = [_vp, C.c_int, _vp, _vp]
        L.qkx_apply_dev.argtypes = [_vp, C.c_int, _vp, _vp]
        L.qkx_spinor_upload.argtypes = [_vp, _vp, _vp]
        L.qkx_spinor_download.argtypes = [_vp, _vp, _vp]
        L.qkx_reCdotXdagY.argtypes = [_vp, _vp, _vp, _dp]
        L.qkx_norm2.argtypes = [_vp, _vp, _dp]
        L.qkx_reCdotXdagY_noalloc.argtypes = [_vp, _vp, C.c_size_t, _dp, _vp]
        L.qkx_X_eq_X_p_aY.argtypes = [_vp, _vp, C.c_double, _vp]
        L.qkx_X_eq_aX_p_Y.argtypes = [_vp, _vp, C.c_double, _vp]
        L.qkx_cg.argtypes = [_vp, _vp, _vp, C.POINTER(SolveInfo)]
        L.qkx_cg_dev.argtypes = [_vp, _vp, _vp, C.POINTER(SolveInfo)]
        L.qkx_invert.argtypes = [_vp, C.POINTER(SolverParams), C.c_int, C.POINTER(_vp),
                                 C.POINTER(_vp), C.POINTER(SolveInfo)]
        L.qkx_invert_dev.argtypes = L.qkx_invert.argtypes
        L.qkx_host_alloc.argtypes = [C.c_size_t]
        L.qkx_host_alloc.restype = _vp
        L.qkx_host_free.argtypes = [_vp]
        L.qkx_host_free.restype = None
        L.qkx_device_alloc.argtypes = [_vp, C.c_size_t]
        L.qkx_device_alloc.restype = _vp
        L.qkx_device_free.argtypes = [_vp, _vp]
        L.qkx_device_free.restype = None
        L.qkx_memcpy_h2d.argtypes = [_vp, _vp, _vp, C.c_size_t]
        L.qkx_memcpy_d2h.argtypes = [_vp, _vp, _vp, C.c_size_t]
        L.qkx_profile_enable.argtypes = [_vp, C.c_int]
        L.qkx_profile_read.argtypes = [_vp, C.POINTER(C.c_longlong), _dp, _dp]
        L.qkx_profile_reset.argtypes = [_vp]
        L.qkx_kernel_launches.argtypes = [_vp]
        L.qkx_kernel_launches.restype = C.c_longlong
        L.qkx_tune.argtypes = [_vp, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp]
        L.qkx_set_tile.argtypes = [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.qkx_tune_table.argtypes = [_vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), _vp, _vp, _vp, _vp]
        L.qkx_sloppy_normal.argtypes = [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_vp),
                                        C.POINTER(_vp)]
        L.qkx_plaquette.argtypes = [_vp, _vp, _dp]
        L.qkx_plaquette_loaded.argtypes = [_vp, C.c_int, _dp]
        L.qkx_project_su3.argtypes = [_vp, _vp]
        L.qkx_ape_smear.argtypes = [_vp, _vp, _vp, C.c_int, C.c_double]
        L.qkx_load_smearing_gauge.argtypes = [_vp, _vp]
        L.qkx_gaussian_smear.argtypes = [_vp, C.c_int, C.POINTER(_vp), C.POINTER(_vp), C.c_int,
                                         C.c_double]
        L.qkx_gaussian_smear_dev.argtypes = L.qkx_gaussian_smear.argtypes
        L.qkx_propagator_absorb.argtypes = [_vp, _vp, C.c_int, C.c_int, _vp]
        L.qkx_propagator.argtypes = [_vp, C.POINTER(SolverParams), C.c_int, C.c_double,
                                     C.POINTER(C.c_int), _vp, C.POINTER(SolveInfo)]
        L.qkx_propagator_dev.argtypes = L.qkx_propagator.argtypes
        L.qkx_ptc_create.argtypes = [_vp, C.POINTER(PtcParams), C.POINTER(_vp)]
        L.qkx_ptc_destroy.argtypes = [_vp]
        L.qkx_ptc_destroy.restype = None
        L.qkx_ptc_num_weights.argtypes = [_vp]
        L.qkx_ptc_num_weights.restype = C.c_long
        L.qkx_ptc_get_weights.argtypes = [_vp, C.c_int, _vp]
        L.qkx_ptc_set_weights.argtypes = [_vp, _vp]
        L.qkx_ptc_apply.argtypes = [_vp, _vp, _vp]
        L.qkx_ptc_loss_grad.argtypes = [_vp, _vp, _vp, _dp, _vp]
        L.qkx_ptc_train.argtypes = [_vp, C.POINTER(PtcTrainParams), C.POINTER(PtcTrainInfo)]
        L.qkx_read_gauge_lime.argtypes = [_vp, C.c_char_p, C.c_int, _vp, C.POINTER(LimeInfo)]
        L.qkx_write_gauge_lime.argtypes = [_vp, C.c_char_p, _vp, C.c_char_p]
        L.qkx_invert_batch.argtypes = [C.POINTER(BatchJob), C.c_int, C.POINTER(SolverParams)]
        L.qkx_momenta.argtypes = [C.c_int, _vp, C.c_int]
        L.qkx_meson_2pt.argtypes = [_vp, _vp, C.c_int, _vp, C.c_int, C.POINTER(C.c_int), _vp]
        L.qkx_meson_2pt_dev.argtypes = L.qkx_meson_2pt.argtypes
        L.qkx_baryon_2pt.argtypes = [_vp, _vp, _vp, C.c_int, C.c_int, C.POINTER(C.c_int), _vp]
        L.qkx_baryon_2pt_dev.argtypes = L.qkx_baryon_2pt.argtypes
        L.qkx_delta_2pt.argtypes = L.qkx_baryon_2pt.argtypes
        L.qkx_delta_2pt_dev.argtypes = L.qkx_baryon_2pt.argtypes
        L.qkx_nucleon_2pt.argtypes = [_vp, _vp, _vp, C.c_int, C.POINTER(C.c_int), _vp]
        L.qkx_nucleon_2pt_dev.argtypes = L.qkx_nucleon_2pt.argtypes
        _lib = L
    return _lib


def check(rc: int) -> int:
    if rc != OK:
        raise QkxError(rc, lib().qkx_last_error().decode())
    return rc


def version() -> str:
    return lib().qkx_version().decode()


@dataclass
class LatticeInfo:
    """The hot-path fields of the reference's struct LatticeInfo (include/qkxTM.h:156-204),
    with the reference's defaults."""
    L: Sequence[int] = (8, 8, 8, 16)
    kappa: float = 0.16
    mu: float = 0.008
    twistSign: int = 1
    boundaryT: int = -1
    tol: float = 1e-1
    maxIter: int = 1000
    reliableDelta: float = 0.1

    def to_c(self) -> Params:
        return Params((C.c_int * 4)(*self.L), self.kappa, self.mu, self.twistSign, self.boundaryT,
                      self.tol, int(self.maxIter), self.reliableDelta)


def _host(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a


class DeviceField:
    """A device spinor in the library's even-odd layout (owned, freed on close)."""

    def __init__(self, lat: "Lattice"):
        self.lat = lat
        self.nbytes = lib().qkx_spinor_bytes(lat.ctx)
        self.ptr = lib().qkx_device_alloc(lat.ctx, self.nbytes)
        if not self.ptr:
            raise QkxError(ERR_NOMEM, "device allocation failed")

    def upload(self, host: np.ndarray) -> "DeviceField":
        h = _host(host)
        check(lib().qkx_spinor_upload(self.lat.ctx, h.ctypes.data, self.ptr))
        check(lib().qkx_sync(self.lat.ctx))
        return self

    def download(self) -> np.ndarray:
        out = np.empty((self.lat.V, 4, 3, 2))
        check(lib().qkx_spinor_download(self.lat.ctx, self.ptr, out.ctypes.data))
        return out

    def close(self):
        if self.ptr:
            lib().qkx_device_free(self.lat.ctx, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Lattice:
    """One lattice on one GPU: gauge field, operators, BLAS and solvers."""

    def __init__(self, info: LatticeInfo, device: int = 0):
        self.info = info
        self.L = tuple(int(v) for v in info.L)
        self.V = int(np.prod(self.L))
        ctx = _vp()
        p = info.to_c()
        check(lib().qkx_create(C.byref(p), device, C.byref(ctx)))
        self.ctx = ctx
        self._owned = weakref.WeakSet()  # networks on this context, closed before it

    def close(self):
        if getattr(self, "ctx", None):
            for o in list(getattr(self, "_owned", ())):
                o.close()
            lib().qkx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_params(self, **kw) -> None:
        for k, v in kw.items():
            setattr(self.info, k, v)
        p = self.info.to_c()
        check(lib().qkx_set_params(self.ctx, C.byref(p)))

    # ------------------------------------------------------------ gauge
    def load_gauge(self, U: np.ndarray, bc_mode: int = LINKS_AS_GIVEN) -> None:
        U = _host(U)
        assert U.size == self.V * 72, "gauge must be [V,4,3,3,2] float64"
        check(lib().qkx_load_gauge(self.ctx, U.ctypes.data, bc_mode))

    def generate_gauge(self, eps: float, seed: int, bc_mode: int = LINKS_APPLY_BC) -> None:
        check(lib().qkx_gauge_generate(self.ctx, eps, seed, bc_mode))

    def read_gauge_lime(self, path: str, bc_mode: int = LINKS_AS_GIVEN, want_host: bool = True):
        """qkxTM_MPI_getGaugeLime: load an ILDG file as the operator's links.
        Returns (Gauge::M array or None, info dict)."""
        U = np.empty((self.V, 4, 3, 3, 2)) if want_host else None
        info = LimeInfo()
        check(lib().qkx_read_gauge_lime(self.ctx, os.fsencode(path), bc_mode,
                                        U.ctypes.data if want_host else None, C.byref(info)))
        return U, {"precision": info.precision, "L": tuple(info.L), "data_offset": info.data_offset,
                   "data_bytes": info.data_bytes, "records": info.records}

    def write_gauge_lime(self, path: str, U: np.ndarray | None = None, message: str = "") -> None:
        """qkxTM_writeGaugeLime: write U (or the operator's links as stored) as an ILDG file."""
        check(lib().qkx_write_gauge_lime(self.ctx, os.fsencode(path), _host(U).ctypes.data if U is not None else None,
                                         message.encode()))

    def download_gauge(self) -> np.ndarray:
        U = np.empty((self.V, 4, 3, 3, 2))
        check(lib().qkx_download_gauge(self.ctx, U.ctypes.data))
        return U

    def compressible(self) -> bool:
        return check_nonneg(lib().qkx_gauge_compressible(self.ctx)) == 1

    # ------------------------------------------------------------ operators
    def apply(self, op: str, psi: np.ndarray) -> np.ndarray:
        psi = _host(psi)
        assert psi.size == self.V * 24, "spinor must be [V,4,3,2] float64"
        out = np.empty((self.V, 4, 3, 2))
        check(lib().qkx_apply(self.ctx, OPS[op], psi.ctypes.data, out.ctypes.data))
        return out

    def apply_dev(self, op: str, src: DeviceField, dst: DeviceField) -> None:
        check(lib().qkx_apply_dev(self.ctx, OPS[op], src.ptr, dst.ptr))

    # reference names (lib/lattice_util.cpp)
    def applyDslash(self, psi): return self.apply("dslash", psi)
    def applyDslashDag(self, psi): return self.apply("dslash_dag", psi)
    def tm(self, psi): return self.apply("tm", psi)
    def tmDag(self, psi): return self.apply("tm_dag", psi)
    def tmDagtm(self, psi): return self.apply("tm_dagtm", psi)
    def Wilson(self, psi): return self.apply("wilson", psi)
    def applyGamma5(self, psi): return self.apply("gamma5", psi)

    def tm_xx(self, psi, parity: str = "EE"):
        return self.apply("tm_xx_" + parity.lower(), psi)

    def tm_xxDagTm_xx(self, psi, parity: str = "EE"):
        return self.apply("tm_xx_dagtm_xx_" + parity.lower(), psi)

    def tm_chiral(self, psi): return self.apply("tm_chiral", psi)

    def tm_xx_chiral(self, psi, parity: str = "EE"):
        return self.apply("tm_xx_chiral_" + parity.lower(), psi)

    def tm_xxDagTm_xx_chiral(self, psi, parity: str = "EE"):
        return self.apply("tm_xx_dagtm_xx_chiral_" + parity.lower(), psi)

    def field(self, host: np.ndarray | None = None) -> DeviceField:
        f = DeviceField(self)
        if host is not None:
            f.upload(host)
        return f

    # ------------------------------------------------------------ BLAS (device fields)
    def reCdotXdagY(self, x: DeviceField, y: DeviceField) -> float:
        r = C.c_double()
        check(lib().qkx_reCdotXdagY(self.ctx, x.ptr, y.ptr, C.byref(r)))
        return r.value

    def norm2(self, x: DeviceField) -> float:
        r = C.c_double()
        check(lib().qkx_norm2(self.ctx, x.ptr, C.byref(r)))
        return r.value

    def X_eq_X_p_aY(self, x: DeviceField, a: float, y: DeviceField) -> None:
        check(lib().qkx_X_eq_X_p_aY(self.ctx, x.ptr, a, y.ptr))

    def X_eq_aX_p_Y(self, x: DeviceField, a: float, y: DeviceField) -> None:
        check(lib().qkx_X_eq_aX_p_Y(self.ctx, x.ptr, a, y.ptr))

    # ------------------------------------------------------------ solvers
    def cg(self, in_: np.ndarray, x: np.ndarray | None = None):
        """CG::operator()(x, in): x += (M^+M)^-1 in, reference stopping rule."""
        in_ = _host(in_)
        x = np.zeros((self.V, 4, 3, 2)) if x is None else _host(x).copy()
        info = SolveInfo()
        rc = lib().qkx_cg(self.ctx, in_.ctypes.data, x.ctypes.data, C.byref(info))
        if rc not in (OK, ERR_NOT_CONVERGED):
            check(rc)
        return x, info

    def invert(self, bs: Sequence[np.ndarray], method: int = SOLVER_CG_EO_MIXED,
               precision: int = PREC_HALF, tol: float = 1e-10, maxIter: int = 10000,
               reliable_delta: float = 0.0, use_graphs: int = 1, strict: bool = True,
               out: Sequence[np.ndarray] | None = None, preconditioner: "Ptc | None" = None):
        """Solve M x_i = b_i to ||b - M x|| / ||b|| <= tol (FP64 true residual).
        `out` may supply the solution arrays (e.g. page-locked buffers)."""
        bs = [_host(b) for b in bs]
        if out is not None:
            xs = list(out)
            for x in xs:
                assert x.dtype == np.float64 and x.flags["C_CONTIGUOUS"] and x.size == self.V * 24
        else:
            xs = [np.empty((self.V, 4, 3, 2)) for _ in bs]
        n = len(bs)
        bp = (_vp * n)(*[b.ctypes.data for b in bs])
        xp = (_vp * n)(*[x.ctypes.data for x in xs])
        sp = SolverParams(method, precision, tol, maxIter, reliable_delta, use_graphs, None,
                          preconditioner.ptr if preconditioner is not None else None)
        info = SolveInfo()
        rc = lib().qkx_invert(self.ctx, C.byref(sp), n, bp, xp, C.byref(info))
        if rc != OK and (strict or rc != ERR_NOT_CONVERGED):
            check(rc)
        return xs, info

    def invert_dev(self, bs: Sequence[DeviceField], xs: Sequence[DeviceField],
                   method: int = SOLVER_CG_EO_MIXED, precision: int = PREC_HALF,
                   tol: float = 1e-10, maxIter: int = 10000, reliable_delta: float = 0.0,
                   use_graphs: int = 1, preconditioner: "Ptc | None" = None) -> SolveInfo:
        n = len(bs)
        bp = (_vp * n)(*[b.ptr for b in bs])
        xp = (_vp * n)(*[x.ptr for x in xs])
        sp = SolverParams(method, precision, tol, maxIter, reliable_delta, use_graphs, None,
                          preconditioner.ptr if preconditioner is not None else None)
        info = SolveInfo()
        check(lib().qkx_invert_dev(self.ctx, C.byref(sp), n, bp, xp, C.byref(info)))
        return info

    # ------------------------------------------------------------ gauge-side stencils
    def plaquette(self, U: np.ndarray | None = None, which: int = LINKS_OPERATOR) -> float:
        """Gauge::calculatePlaquette of host links U, or of a field the context holds."""
        r = C.c_double()
        if U is not None:
            check(lib().qkx_plaquette(self.ctx, _host(U).ctypes.data, C.byref(r)))
        else:
            check(lib().qkx_plaquette_loaded(self.ctx, which, C.byref(r)))
        return r.value

    calculatePlaquette = plaquette

    def project_su3(self, U: np.ndarray) -> np.ndarray:
        """qcd_projectSU33d on the spatial links of a copy of U."""
        U = _host(U).copy()
        check(lib().qkx_project_su3(self.ctx, U.ctypes.data))
        return U

    def APE_smearing(self, U_in: np.ndarray, nsmear: int = 20, alpha: float = 0.5,
                     out: np.ndarray | None = None, download: bool = True) -> np.ndarray | None:
        """Gauge::APE_smearing of U_in; the result also becomes the smearing links.
        Returns the smeared field (out, or a new array; None with download=False);
        nsmear == 0 leaves out as it was."""
        if not download:
            check(lib().qkx_ape_smear(self.ctx, _host(U_in).ctypes.data, None, nsmear, alpha))
            return None
        out = np.zeros_like(_host(U_in)) if out is None else out
        check(lib().qkx_ape_smear(self.ctx, _host(U_in).ctypes.data, out.ctypes.data, nsmear, alpha))
        return out

    def load_smearing_gauge(self, U: np.ndarray) -> None:
        check(lib().qkx_load_smearing_gauge(self.ctx, _host(U).ctypes.data))

    def Gaussian_smearing(self, psis: Sequence[np.ndarray], nsmear: int = 50, alpha: float = 4.0,
                          out: Sequence[np.ndarray] | None = None) -> list:
        """Vector::Gaussian_smearing of every field of psis with the smearing links."""
        psis = [_host(p) for p in psis]
        outs = [np.zeros_like(p) for p in psis] if out is None else list(out)
        n = len(psis)
        ip = (_vp * n)(*[p.ctypes.data for p in psis])
        op = (_vp * n)(*[o.ctypes.data for o in outs])
        check(lib().qkx_gaussian_smear(self.ctx, n, ip, op, nsmear, alpha))
        return outs

    def Gaussian_smearing_dev(self, src: Sequence[DeviceField], dst: Sequence[DeviceField],
                              nsmear: int = 50, alpha: float = 4.0) -> None:
        n = len(src)
        ip = (_vp * n)(*[f.ptr for f in src])
        op = (_vp * n)(*[f.ptr for f in dst])
        check(lib().qkx_gaussian_smear_dev(self.ctx, n, ip, op, nsmear, alpha))

    def absorbVector(self, prop: np.ndarray, phi: np.ndarray, nu: int, c2: int) -> None:
        """Propagator::absorbVector: prop[x, mu, nu, c1, c2] = phi[x, mu, c1] (prop in place)."""
        assert prop.dtype == np.float64 and prop.flags["C_CONTIGUOUS"] and prop.size == self.V * 288
        check(lib().qkx_propagator_absorb(self.ctx, _host(phi).ctypes.data, nu, c2, prop.ctypes.data))

    def propagator(self, x_src=(0, 0, 0, 0), nsmear: int = 50, alpha: float = 4.0,
                   method: int = SOLVER_CG_EO_MIXED, precision: int = PREC_HALF, tol: float = 1e-10,
                   maxIter: int = 10000, reliable_delta: float = 0.0, use_graphs: int = 1,
                   out: np.ndarray | None = None):
        """The smeared-source propagator [V, 4, 4, 3, 3, 2] at x_src; returns (prop, info)."""
        prop = np.empty((self.V, 4, 4, 3, 3, 2)) if out is None else out
        assert prop.dtype == np.float64 and prop.flags["C_CONTIGUOUS"] and prop.size == self.V * 288
        sp = SolverParams(method, precision, tol, maxIter, reliable_delta, use_graphs)
        info = SolveInfo()
        rc = lib().qkx_propagator(self.ctx, C.byref(sp), nsmear, alpha, (C.c_int * 4)(*x_src),
                                  prop.ctypes.data, C.byref(info))
        check(rc)
        return prop, info

    def propagator_dev(self, prop_ptr: int, x_src=(0, 0, 0, 0), nsmear: int = 50, alpha: float = 4.0,
                       method: int = SOLVER_CG_EO_MIXED, precision: int = PREC_HALF, tol: float = 1e-10,
                       maxIter: int = 10000, reliable_delta: float = 0.0,
                       use_graphs: int = 1) -> SolveInfo:
        """The same into device memory at prop_ptr (V * 2304 bytes, host layout); asynchronous."""
        sp = SolverParams(method, precision, tol, maxIter, reliable_delta, use_graphs)
        info = SolveInfo()
        check(lib().qkx_propagator_dev(self.ctx, C.byref(sp), nsmear, alpha, (C.c_int * 4)(*x_src),
                                       prop_ptr, C.byref(info)))
        return info

    # ------------------------------------------------------------ two-point functions
    def meson_2pt(self, prop, ops=tuple(range(10)), Q_sq: int = 0, x_src=(0, 0, 0, 0), device: bool = False):
        """Meson::contract + fourier(FORWARD) for the operators ops: [nop, Lt, Nmom, 2].
        prop is a host array, or with device=True a device pointer (int)."""
        ops = list(ops)
        nmom = len(momenta(Q_sq))
        out = np.zeros((len(ops), self.info.L[3], nmom, 2))
        f = lib().qkx_meson_2pt_dev if device else lib().qkx_meson_2pt
        ptr = prop if device else _host(prop).ctypes.data
        check(f(self.ctx, ptr, len(ops), (C.c_int * len(ops))(*ops), Q_sq, (C.c_int * 4)(*x_src), out.ctypes.data))
        return out

    def baryon_2pt(self, prop1, prop2, op: int, Q_sq: int = 0, x_src=(0, 0, 0, 0), device: bool = False):
        """Baryon::contract(prop1, prop2, op) + fourier(FORWARD): [Lt, Nmom, 4, 4, 2]."""
        nmom = len(momenta(Q_sq))
        out = np.zeros((self.info.L[3], nmom, 4, 4, 2))
        f = lib().qkx_baryon_2pt_dev if device else lib().qkx_baryon_2pt
        p1 = prop1 if device else _host(prop1).ctypes.data
        p2 = prop2 if device else _host(prop2).ctypes.data
        check(f(self.ctx, p1, p2, op, Q_sq, (C.c_int * 4)(*x_src), out.ctypes.data))
        return out

    def delta_2pt(self, prop1, prop2, op: int, Q_sq: int = 0, x_src=(0, 0, 0, 0), device: bool = False):
        """Baryon_Dec::contract(prop1, prop2, op) + fourier(FORWARD): [Lt, Nmom, 3, 4, 4, 2]
        (op 0 DELTA_ISO1, 1 DELTA_ISO1O2)."""
        nmom = len(momenta(Q_sq))
        out = np.zeros((self.info.L[3], nmom, 3, 4, 4, 2))
        f = lib().qkx_delta_2pt_dev if device else lib().qkx_delta_2pt
        p1 = prop1 if device else _host(prop1).ctypes.data
        p2 = prop2 if device else _host(prop2).ctypes.data
        check(f(self.ctx, p1, p2, op, Q_sq, (C.c_int * 4)(*x_src), out.ctypes.data))
        return out

    def nucleon_2pt(self, prop1, prop2, Q_sq: int = 0, x_src=(0, 0, 0, 0), device: bool = False):
        """contractNucleon(prop1, prop2, ..., Q_sq, x_src) (lib/lattice_util.cpp:3374): the
        numbers it prints, as [Lt, Nmom, 4, 4, 2]."""
        nmom = len(momenta(Q_sq))
        out = np.zeros((self.info.L[3], nmom, 4, 4, 2))
        f = lib().qkx_nucleon_2pt_dev if device else lib().qkx_nucleon_2pt
        p1 = prop1 if device else _host(prop1).ctypes.data
        p2 = prop2 if device else _host(prop2).ctypes.data
        check(f(self.ctx, p1, p2, Q_sq, (C.c_int * 4)(*x_src), out.ctypes.data))
        return out

    # ------------------------------------------------------------ profiling
    def profile(self, on: bool) -> None:
        check(lib().qkx_profile_enable(self.ctx, int(on)))

    def profile_read(self):
        n, ms, by = C.c_longlong(), C.c_double(), C.c_double()
        check(lib().qkx_profile_read(self.ctx, C.byref(n), C.byref(ms), C.byref(by)))
        return n.value, ms.value, by.value

    def profile_reset(self) -> None:
        check(lib().qkx_profile_reset(self.ctx))

    def sync(self) -> None:
        check(lib().qkx_sync(self.ctx))

    def tune(self, precision: int = PREC_HALF, nrhs: int = 12):
        """Autotune the inner hop; returns (rhs_per_thread, threads_per_block, ms_per_hop)."""
        nr, nt, ms = C.c_int(), C.c_int(), C.c_double()
        check(lib().qkx_tune(self.ctx, precision, nrhs, C.byref(nr), C.byref(nt), C.byref(ms)))
        return nr.value, nt.value, ms.value

    def set_tile(self, precision: int, nrhs: int, tile) -> None:
        """Use this hop tile (rhs_per_thread, threads_per_block[, kind]) for later mixed solves of
        this precision and batch size instead of the tuned one."""
        t = tuple(tile) + (0,) * (3 - len(tile))
        check(lib().qkx_set_tile(self.ctx, precision, nrhs, int(t[0]), int(t[1]), int(t[2])))

    def tune_table(self, precision: int = PREC_HALF, nrhs: int = 12) -> list:
        """Every tile timed by the last tuning of (precision, nrhs): dicts with the tile
        (rhs_per_thread, threads_per_block, kind) and its ms per hop."""
        n = C.c_int()
        check(lib().qkx_tune_table(self.ctx, precision, nrhs, 0, C.byref(n), None, None, None, None))
        k = n.value
        nr, nt, kd = (C.c_int * max(k, 1))(), (C.c_int * max(k, 1))(), (C.c_int * max(k, 1))()
        ms = (C.c_double * max(k, 1))()
        check(lib().qkx_tune_table(self.ctx, precision, nrhs, k, C.byref(n), nr, nt, kd, ms))
        return [{"tile": [nr[i], nt[i], kd[i]], "ms_per_hop": ms[i]} for i in range(k)]

    def sloppy_normal(self, psis: Sequence[np.ndarray], precision: int = PREC_HALF, tile=(0, 0, 0)) -> list:
        """tm_xxDagTm_xx(EE) of every field as the mixed solver's inner iteration computes it: the
        even sites rounded to the sloppy precision and the four sloppy hops with the given tile
        (rhs_per_thread, threads_per_block[, kind]); (0, 0, 0) = the tuned tile.  Odd sites of the
        results are zero."""
        psis = [_host(p) for p in psis]
        outs = [np.zeros_like(p) for p in psis]
        n = len(psis)
        ip = (_vp * n)(*[p.ctypes.data for p in psis])
        op = (_vp * n)(*[o.ctypes.data for o in outs])
        t = tuple(tile) + (0,) * (3 - len(tile))
        check(lib().qkx_sloppy_normal(self.ctx, precision, n, int(t[0]), int(t[1]), int(t[2]), ip, op))
        return outs

    def kernel_launches(self) -> int:
        return int(lib().qkx_kernel_launches(self.ctx))

    def stream(self) -> int:
        return int(lib().qkx_stream(self.ctx) or 0)


class Ptc:
    """The learned preconditioner: a linear gauge-covariant parallel-transport convolution
    network on the lattice's links (no reference counterpart).  channels are the widths per
    colour, first and last 4 (the spins)."""

    def __init__(self, lat: Lattice, channels=(4, 16, 16, 16, 4), seed: int = 1, init_scale: float = 0.1,
                 tensor_cores: bool = True):
        self.lat = lat
        self.channels = tuple(channels)
        nl = len(channels) - 1
        p = PtcParams(nl, (C.c_int * (PTC_MAX_LAYERS + 1))(*channels), seed, init_scale, int(tensor_cores))
        self.ptr = _vp()
        check(lib().qkx_ptc_create(lat.ctx, C.byref(p), C.byref(self.ptr)))
        self.nw = int(lib().qkx_ptc_num_weights(self.ptr))
        lat._owned.add(self)

    def close(self):
        # a network lives on its lattice's context: the lattice closes it first when it closes
        if getattr(self, "ptr", None) and self.ptr.value and getattr(self.lat, "ctx", None):
            lib().qkx_ptc_destroy(self.ptr)
        self.ptr = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def weights(self, which: int = 0) -> np.ndarray:
        """[nweights, 2]: which = 0 the FP32 master weights, 1 the BF16 weights the kernels use."""
        w = np.empty((self.nw, 2))
        check(lib().qkx_ptc_get_weights(self.ptr, which, w.ctypes.data))
        return w

    def set_weights(self, w: np.ndarray) -> None:
        w = _host(w)
        assert w.size == 2 * self.nw
        check(lib().qkx_ptc_set_weights(self.ptr, w.ctypes.data))

    def apply(self, psi: np.ndarray) -> np.ndarray:
        out = np.empty((self.lat.V, 4, 3, 2))
        check(lib().qkx_ptc_apply(self.ptr, _host(psi).ctypes.data, out.ctypes.data))
        return out

    def loss_grad(self, r: np.ndarray, e: np.ndarray, grad: bool = True):
        """(|N(r) - e|^2 / |e|^2, dL/dW^* as [nweights, 2] or None)."""
        loss = C.c_double()
        g = np.empty((self.nw, 2)) if grad else None
        check(lib().qkx_ptc_loss_grad(self.ptr, _host(r).ctypes.data, _host(e).ctypes.data, C.byref(loss),
                                      g.ctypes.data if grad else None))
        return loss.value, g

    def train(self, n_solves: int = 64, steps: int = 2000, lr: float = 2e-3, solve_tol: float = 1e-6,
              seed: int = 7) -> dict:
        tp = PtcTrainParams(n_solves, steps, lr, solve_tol, seed)
        info = PtcTrainInfo()
        check(lib().qkx_ptc_train(self.ptr, C.byref(tp), C.byref(info)))
        return info.as_dict()


def invert_batch(jobs, method: int = SOLVER_CG_EO_MIXED, precision: int = PREC_HALF, tol: float = 1e-10,
                 maxIter: int = 10000, use_graphs: int = 1):
    """Run many solves on several lattices concurrently (qkx_invert_batch).
    jobs: list of (Lattice, [DeviceField b], [DeviceField x], mu list or None).
    Returns a list of dicts with the status, latency (s from the batch start) and solve info."""
    arr = (BatchJob * len(jobs))()
    keep = []
    for j, (lat, bs, xs, mus) in zip(arr, jobs):
        bp = (_vp * len(bs))(*[b.ptr for b in bs])
        xp = (_vp * len(xs))(*[x.ptr for x in xs])
        mp = (C.c_double * len(mus))(*mus) if mus is not None else None
        keep += [bp, xp, mp]
        j.ctx, j.nrhs, j.b_dev, j.x_dev = lat.ctx, len(bs), bp, xp
        j.mu = C.cast(mp, C.POINTER(C.c_double)) if mp is not None else None
    sp = SolverParams(method, precision, tol, maxIter, 0.0, use_graphs, None, None)
    rc = lib().qkx_invert_batch(arr, len(jobs), C.byref(sp))
    out = [{"status": j.status, "latency": j.latency, "info": j.info.as_dict(), "message": j.message.decode()}
           for j in arr]
    if rc != OK:
        check(rc)
    return out


MESONS = ["ONE", "G5", "G1", "G2", "G3", "G4", "G5G1", "G5G2", "G5G3", "G5G4"]
BARYONS = ["NTN", "NTR", "RTN", "RTR"]
DELTAS = ["ISO1", "ISO1O2"]


def momenta(Q_sq: int) -> np.ndarray:
    """createMomenta (lib/contractions.cpp:37) as [Nmom, 3]."""
    n = lib().qkx_momenta(Q_sq, None, 0)
    if n < 0:
        check(n)
    m = np.zeros((n, 3), dtype=np.int32)
    lib().qkx_momenta(Q_sq, m.ctypes.data, n)
    return m


def pinned_array(shape) -> np.ndarray:
    """A float64 numpy array in page-locked host memory (freed with the array)."""
    n = int(np.prod(shape))
    ptr = lib().qkx_host_alloc(n * 8)
    if not ptr:
        raise QkxError(ERR_NOMEM, "page-locked host allocation failed")
    buf = (C.c_double * n).from_address(ptr)
    arr = np.ctypeslib.as_array(buf).reshape(shape)
    import weakref
    weakref.finalize(buf, lib().qkx_host_free, ptr)
    return arr


def check_nonneg(rc: int) -> int:
    if rc < 0:
        check(rc)
    return rc
