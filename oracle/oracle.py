"""ctypes bindings for the CPU oracle (oracle/liboracle.so) and for the
reference's own sources compiled into oracle/_ref/libqkxref.so.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py`` -- always as the checker or the
timed CPU baseline, never as part of the product path.

Arrays are numpy float64 in the reference's host layouts:
spinor ``[V, 4, 3, 2]`` (Vector::M, include/lattice_util.h:90) and gauge
``[V, 4, 3, 3, 2]`` (Gauge::M, include/lattice_util.h:198), site order
x fastest (LEXIC, include/qkxTM.h:130).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libqkxref.so")
# where the reference sources lie (only the build of the pin and the fixture script read them)
REF_SRC = os.environ.get("QKX_REFERENCE_SRC", "/root/reference")

UKQCD, CHIRAL = 0, 1
EO, OE, OO, EE = 0, 1, 2, 3

# operator ids of ref_shim.cpp
REF_OPS = {
    "dslash": 0, "dslash_dag": 1, "tm": 2, "tm_dag": 3, "tm_dagtm": 4, "wilson": 5,
    "tm_xx_ee": 6, "tm_xx_oo": 7, "tm_xx_dagtm_xx_ee": 8, "tm_xx_dagtm_xx_oo": 9,
    "dslash_chiral": 10, "tm_chiral": 11, "tm_xx_chiral_ee": 12, "tm_xx_chiral_oo": 13,
    "tm_xx_dagtm_xx_chiral_ee": 14, "tm_xx_dagtm_xx_chiral_oo": 15, "gamma5": 16,
    "gamma5_chiral": 17, "twist": 18, "twist_inv": 19, "twist_dag": 20, "twist_dag_inv": 21,
    "twist_inv_chiral": 22, "dslash_xx_eo": 23, "dslash_xx_oe": 24,
    "rotate_chiral_to_ukqcd": 25, "dslash_xx_chiral_eo": 26, "dslash_xx_chiral_oe": 27,
}


class OrcParams(C.Structure):
    _fields_ = [("L", C.c_int * 4), ("kappa", C.c_double), ("mu", C.c_double),
                ("twistSign", C.c_int), ("boundaryT", C.c_int), ("tol", C.c_double),
                ("maxIter", C.c_int)]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def _L(L):
    return (C.c_int * 4)(*L)


def build(ref: bool = True) -> None:
    """Compile the oracle (and the reference build when its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref and os.path.isdir(os.path.join(REF_SRC, "lib")):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "ref"), f"REF={REF_SRC}"],
                       check=True)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        _lib = C.CDLL(ORACLE_SO)
        L = _lib
        L.orc_volume.restype = C.c_long
        L.orc_gauge_random.argtypes = [_ip, C.c_double, C.c_ulonglong, _dp]
        L.orc_spinor_gaussian.argtypes = [_ip, C.c_ulonglong, _dp]
        L.orc_spinor_point.argtypes = [_ip, _ip, C.c_int, C.c_int, _dp]
        L.orc_plaquette.argtypes = [_ip, _dp]
        L.orc_plaquette.restype = C.c_double
        L.orc_re_dot.restype = C.c_double
        L.orc_re_dot.argtypes = [C.c_long, _dp, _dp]
        L.orc_norm2.restype = C.c_double
        L.orc_norm2.argtypes = [C.c_long, _dp]
        L.orc_axpy.argtypes = [C.c_long, C.c_double, _dp, _dp]
        L.orc_xpay.argtypes = [C.c_long, C.c_double, _dp, _dp]
        L.orc_cg.restype = C.c_int
        L.orc_plaquette_ref.argtypes = [_ip, _dp]
        L.orc_plaquette_ref.restype = C.c_double
        L.orc_su3_project_many.argtypes = [C.c_long, _dp]
        L.orc_ape_smear.argtypes = [_ip, _dp, _dp, C.c_int, C.c_double]
        L.orc_gaussian_smear.argtypes = [_ip, _dp, _dp, _dp, C.c_int, C.c_double]
        L.orc_absorb_vector.argtypes = [C.c_long, _dp, C.c_int, C.c_int, _dp]
        L.orc_momenta.argtypes = [C.c_int, _ip, C.c_int]
        L.orc_meson_2pt.argtypes = [_ip, _dp, C.c_int, C.c_int, _ip, _dp]
        L.orc_baryon_2pt.argtypes = [_ip, _dp, _dp, C.c_int, C.c_int, _ip, _dp]
        L.orc_delta_2pt.argtypes = [_ip, _dp, _dp, C.c_int, C.c_int, _ip, _dp]
        L.orc_nucleon_2pt.argtypes = [_ip, _dp, _dp, C.c_int, _ip, _dp]
        L.orc_ptc_nweights.argtypes = [C.c_int, _ip]
        L.orc_ptc_nweights.restype = C.c_long
        L.orc_ptc_forward.argtypes = [_ip, _dp, C.c_int, _ip, _dp, _dp, _dp, _dp]
        L.orc_ptc_loss_grad.argtypes = [_ip, _dp, C.c_int, _ip, _dp, _dp, _dp, _dp]
        L.orc_ptc_loss_grad.restype = C.c_double
        L.orc_ptc_act_bf16.argtypes = [C.c_int]
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        _ref = C.CDLL(REF_SO)
        _ref.ref_apply.restype = C.c_int
        _ref.ref_apply.argtypes = [C.c_int, _ip, C.c_double, C.c_double, C.c_int, _dp, _dp, _dp]
        _ref.ref_blas.restype = C.c_double
        _ref.ref_blas.argtypes = [C.c_int, _ip, C.c_double, _dp, _dp]
        _ref.ref_cg.argtypes = [_ip, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int,
                                _dp, _dp, _dp]
        _ref.ref_apply_bc.argtypes = [_ip, C.c_int, _dp]
        _ref.ref_plaquette.argtypes = [_ip, _dp]
        _ref.ref_plaquette.restype = C.c_double
        _ref.ref_project_su3.argtypes = [_ip, _dp]
        _ref.ref_ape_smear.argtypes = [_ip, _dp, _dp, C.c_int, C.c_double]
        _ref.ref_gaussian_smear.argtypes = [_ip, _dp, _dp, _dp, C.c_int, C.c_double]
        _ref.ref_absorb_vector.argtypes = [_ip, _dp, C.c_int, C.c_int, _dp]
        _ref.ref_read_gauge_lime.argtypes = [C.c_char_p, _ip, _dp]
        _ref.ref_write_gauge_lime.argtypes = [C.c_char_p, _ip, _dp, C.c_char_p]
        _ref.ref_meson_2pt.argtypes = [_ip, _dp, C.c_int, C.c_int, _ip, _dp]
        _ref.ref_delta_2pt.argtypes = [_ip, _dp, _dp, C.c_int, C.c_int, _ip, _dp]
        _ref.ref_contract_nucleon.argtypes = [_ip, _dp, _dp, C.c_int, _ip, C.c_char_p]
        _ref.ref_baryon_2pt.argtypes = [_ip, _dp, _dp, C.c_int, C.c_int, _ip, _dp]
        _ref.ref_propagator.argtypes = [_ip, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int,
                                        _dp, _dp, C.c_int, C.c_double, C.c_long, _dp]
    return _ref


def volume(L) -> int:
    return int(L[0]) * L[1] * L[2] * L[3]


def params(L, kappa, mu, twistSign=1, boundaryT=-1, tol=1e-10, maxIter=1000) -> OrcParams:
    return OrcParams(_L(L), kappa, mu, twistSign, boundaryT, tol, maxIter)


# ---------------------------------------------------------------- inputs
def gauge_random(L, eps, seed) -> np.ndarray:
    U = np.empty((volume(L), 4, 3, 3, 2))
    lib().orc_gauge_random(_L(L), eps, seed, _ptr(U))
    return U


def gauge_unit(L) -> np.ndarray:
    U = np.empty((volume(L), 4, 3, 3, 2))
    lib().orc_gauge_unit(_L(L), _ptr(U))
    return U


def spinor_gaussian(L, seed) -> np.ndarray:
    v = np.empty((volume(L), 4, 3, 2))
    lib().orc_spinor_gaussian(_L(L), seed, _ptr(v))
    return v


def spinor_point(L, x, spin, colour) -> np.ndarray:
    v = np.empty((volume(L), 4, 3, 2))
    lib().orc_spinor_point(_L(L), (C.c_int * 4)(*x), spin, colour, _ptr(v))
    return v


def plaquette(L, U) -> float:
    return lib().orc_plaquette(_L(L), _ptr(U))


def apply_bc(L, U, boundaryT=-1) -> np.ndarray:
    U = U.copy()
    lib().orc_apply_bc(_L(L), boundaryT, _ptr(U))
    return U


# ---------------------------------------------------------------- operators
def apply(op: str, L, U, psi, kappa=0.16, mu=0.01, twistSign=1) -> np.ndarray:
    """Oracle operator by the same names as REF_OPS."""
    lb = lib()
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    out = np.empty_like(psi)
    p = params(L, kappa, mu, twistSign)
    pp = C.byref(p)
    Lc = _L(L)
    basis = CHIRAL if ("chiral" in op and op != "rotate_chiral_to_ukqcd") else UKQCD
    base = op if op == "rotate_chiral_to_ukqcd" else op.replace("_chiral", "")
    if base == "dslash":
        lb.orc_dslash(Lc, _ptr(U), _ptr(psi), _ptr(out), 0, basis)
    elif base == "dslash_dag":
        lb.orc_dslash(Lc, _ptr(U), _ptr(psi), _ptr(out), 1, basis)
    elif base in ("dslash_xx_eo", "dslash_xx_oe"):
        lb.orc_dslash_xx(Lc, _ptr(U), _ptr(psi), _ptr(out), EO if base.endswith("eo") else OE, basis)
    elif base == "tm":
        lb.orc_tm(pp, _ptr(U), _ptr(psi), _ptr(out), basis)
    elif base == "tm_dag":
        lb.orc_tm_dag(pp, _ptr(U), _ptr(psi), _ptr(out), basis)
    elif base == "tm_dagtm":
        lb.orc_tm_dagtm(pp, _ptr(U), _ptr(psi), _ptr(out), basis)
    elif base == "wilson":
        lb.orc_wilson(pp, _ptr(U), _ptr(psi), _ptr(out))
    elif base in ("tm_xx_ee", "tm_xx_oo"):
        lb.orc_tm_xx(pp, _ptr(U), _ptr(psi), _ptr(out), EE if base.endswith("ee") else OO, basis)
    elif base in ("tm_xx_dagtm_xx_ee", "tm_xx_dagtm_xx_oo"):
        lb.orc_tm_xx_dagtm_xx(pp, _ptr(U), _ptr(psi), _ptr(out),
                              EE if base.endswith("ee") else OO, basis)
    elif base == "gamma5":
        lb.orc_gamma5(Lc, _ptr(psi), _ptr(out), basis)
    elif base in ("twist", "twist_inv", "twist_dag", "twist_dag_inv"):
        lb.orc_twist(pp, _ptr(psi), _ptr(out), int("dag" in base), int("inv" in base), basis)
    elif base == "rotate_chiral_to_ukqcd":
        out[...] = psi
        lb.orc_rotate_chiral_to_ukqcd(Lc, _ptr(out))
    else:
        raise ValueError(op)
    return out


def ref_apply(op: str, L, U, psi, kappa=0.16, mu=0.01, twistSign=1) -> np.ndarray:
    """The reference's own operator (needs oracle/_ref/libqkxref.so)."""
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    out = np.empty_like(psi)
    rc = ref().ref_apply(REF_OPS[op], _L(L), kappa, mu, twistSign, _ptr(U), _ptr(psi), _ptr(out))
    if rc != 0:
        raise ValueError(op)
    return out


# ---------------------------------------------------------------- BLAS / CG
def re_dot(x, y) -> float:
    return lib().orc_re_dot(x.shape[0], _ptr(x), _ptr(y))


def norm2(x) -> float:
    return lib().orc_norm2(x.shape[0], _ptr(x))


def axpy(a, y, x) -> None:
    lib().orc_axpy(x.shape[0], a, _ptr(y), _ptr(x))


def xpay(a, y, x) -> None:
    lib().orc_xpay(x.shape[0], a, _ptr(y), _ptr(x))


def cg(L, U, b, kappa, mu, twistSign=1, tol=1e-10, maxIter=1000, x0=None):
    """CG on M^dag M (lib/solvers.cpp:16-81).  Returns (x, iterations, r2 trace)."""
    x = np.zeros_like(b) if x0 is None else x0.copy()
    p = params(L, kappa, mu, twistSign, -1, tol, maxIter)
    trace = np.zeros(maxIter + 1)
    lib().orc_cg.argtypes = [C.POINTER(OrcParams), _dp, _dp, _dp, _dp, C.c_int]
    k = lib().orc_cg(C.byref(p), _ptr(U), _ptr(np.ascontiguousarray(b)), _ptr(x), _ptr(trace),
                     maxIter + 1)
    return x, k, trace[: k + 1]


def ref_cg(L, U, b, kappa, mu, twistSign=1, tol=1e-10, maxIter=1000, x0=None):
    x = np.zeros_like(b) if x0 is None else x0.copy()
    ref().ref_cg(_L(L), kappa, mu, twistSign, tol, maxIter, _ptr(U),
                 _ptr(np.ascontiguousarray(b)), _ptr(x))
    return x


def ref_read_gauge_lime(path, L) -> np.ndarray:
    """qkxTM_MPI_getGaugeLime (lib/read_conf_lime.cpp:111-245), the reference compiled with
    the LIME and MPI-IO stand-ins of oracle/ref: the file's links as Gauge::M."""
    U = np.zeros((volume(L), 4, 3, 3, 2))
    rc = ref().ref_read_gauge_lime(os.fsencode(str(path)), _L(L), _ptr(U))
    if rc != 0:
        raise RuntimeError(f"reference LIME reader returned {rc}")
    return U


def ref_write_gauge_lime(path, L, U: np.ndarray, message: bytes) -> None:
    """qkxTM_writeGaugeLime (lib/write_conf_lime.cpp:49-199): U as an ILDG file."""
    U = np.ascontiguousarray(U, dtype=np.float64)
    rc = ref().ref_write_gauge_lime(os.fsencode(str(path)), _L(L), _ptr(U), message)
    if rc != 0:
        raise RuntimeError(f"reference LIME writer returned {rc}")


def rel_err(a, b) -> float:
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


# ---------------------------------------------------------------- smearing / propagator
def plaquette_ref(L, U) -> float:
    """Gauge::calculatePlaquette restated (lib/lattice_util.cpp:923)."""
    return lib().orc_plaquette_ref(_L(L), _ptr(np.ascontiguousarray(U)))


def su3_project(m) -> np.ndarray:
    """qcd_projectSU33d restated (lib/blas.cpp:6) on a stack of 3x3 matrices [..., 3, 3, 2]."""
    m = np.ascontiguousarray(m, dtype=np.float64).copy()
    lib().orc_su3_project_many(m.size // 18, _ptr(m))
    return m


def ape_smear(L, U, nsmear, alpha, out=None) -> np.ndarray:
    """Gauge::APE_smearing restated (lib/lattice_util.cpp:948)."""
    out = np.zeros_like(U) if out is None else out.copy()
    lib().orc_ape_smear(_L(L), _ptr(np.ascontiguousarray(U)), _ptr(out), nsmear, alpha)
    return out


def gaussian_smear(L, U, psi, nsmear, alpha, out=None) -> np.ndarray:
    """Vector::Gaussian_smearing restated (lib/lattice_util.cpp:1080)."""
    out = np.zeros_like(psi) if out is None else out.copy()
    lib().orc_gaussian_smear(_L(L), _ptr(np.ascontiguousarray(U)), _ptr(np.ascontiguousarray(psi)),
                             _ptr(out), nsmear, alpha)
    return out


def absorb_vector(phi, nu, c2, prop) -> None:
    """Propagator::absorbVector restated (lib/lattice_util.cpp:2073), prop updated in place."""
    lib().orc_absorb_vector(phi.shape[0], _ptr(np.ascontiguousarray(phi)), nu, c2, _ptr(prop))


def ref_plaquette(L, U) -> float:
    return ref().ref_plaquette(_L(L), _ptr(np.ascontiguousarray(U)))


def ref_project_su3(L, U) -> np.ndarray:
    U = np.ascontiguousarray(U, dtype=np.float64).copy()
    ref().ref_project_su3(_L(L), _ptr(U))
    return U


def ref_ape_smear(L, U, nsmear, alpha, out=None) -> np.ndarray:
    out = np.zeros_like(U) if out is None else out.copy()
    ref().ref_ape_smear(_L(L), _ptr(np.ascontiguousarray(U)), _ptr(out), nsmear, alpha)
    return out


def ref_gaussian_smear(L, U, psi, nsmear, alpha, out=None) -> np.ndarray:
    out = np.zeros_like(psi) if out is None else out.copy()
    ref().ref_gaussian_smear(_L(L), _ptr(np.ascontiguousarray(U)), _ptr(np.ascontiguousarray(psi)),
                             _ptr(out), nsmear, alpha)
    return out


def ref_absorb_vector(L, phi, nu, c2, prop) -> None:
    ref().ref_absorb_vector(_L(L), _ptr(np.ascontiguousarray(phi)), nu, c2, _ptr(prop))


def ref_propagator(L, U, U_smear, kappa, mu, nsmear, alpha, src=0, twistSign=1, tol=1e-10,
                   maxIter=1000) -> np.ndarray:
    """The propagator loop of bin/test_invert_prop.cpp:83-97 run by the reference."""
    prop = np.zeros((volume(L), 4, 4, 3, 3, 2))
    ref().ref_propagator(_L(L), kappa, mu, twistSign, tol, maxIter, _ptr(np.ascontiguousarray(U)),
                         _ptr(np.ascontiguousarray(U_smear)), nsmear, alpha, src, _ptr(prop))
    return prop


# ---------------------------------------------------------------- learned preconditioner (PTC network)
def ptc_nweights(ch) -> int:
    """Complex weights of a PTC network with channel widths ch (9 paths per layer)."""
    return int(lib().orc_ptc_nweights(len(ch) - 1, (C.c_int * len(ch))(*ch)))


def ptc_forward(L, U, ch, W, x, bf16=False) -> np.ndarray:
    """N(x) for x [V, ch[0], 3, 2]; W complex weights as float64 [nweights, 2].  bf16: the
    hidden activations rounded to BF16 as the GPU stores them (arithmetic FP64)."""
    V = volume(L)
    out = np.empty((V, ch[-1], 3, 2))
    lib().orc_ptc_act_bf16(1 if bf16 else 0)
    try:
        lib().orc_ptc_forward(_L(L), _ptr(np.ascontiguousarray(U)), len(ch) - 1, (C.c_int * len(ch))(*ch),
                              _ptr(np.ascontiguousarray(W)), _ptr(np.ascontiguousarray(x)), _ptr(out), None)
    finally:
        lib().orc_ptc_act_bf16(0)
    return out


def ptc_loss_grad(L, U, ch, W, r, e, grad=True, bf16=False):
    """(|N(r) - e|^2 / |e|^2, dL/dW^* as [nweights, 2] or None); bf16 as in ptc_forward, for
    the activation gradients between layers too."""
    g = np.zeros_like(W) if grad else None
    lib().orc_ptc_act_bf16(1 if bf16 else 0)
    try:
        loss = lib().orc_ptc_loss_grad(_L(L), _ptr(np.ascontiguousarray(U)), len(ch) - 1,
                                       (C.c_int * len(ch))(*ch), _ptr(np.ascontiguousarray(W)),
                                       _ptr(np.ascontiguousarray(r)), _ptr(np.ascontiguousarray(e)),
                                       _ptr(g) if grad else None)
    finally:
        lib().orc_ptc_act_bf16(0)
    return loss, g


# ---------------------------------------------------------------- contractions
MESONS = ["ONE", "G5", "G1", "G2", "G3", "G4", "G5G1", "G5G2", "G5G3", "G5G4"]
BARYONS = ["NTN", "NTR", "RTN", "RTR"]


def momenta(Q_sq) -> np.ndarray:
    """createMomenta (lib/contractions.cpp:37) as [Nmom, 3]."""
    buf = np.zeros(3000, dtype=np.int32)
    n = lib().orc_momenta(Q_sq, buf.ctypes.data_as(_ip), 1000)
    return buf[:3 * n].reshape(n, 3).copy()


def meson_2pt(L, prop, op, Q_sq=0, x_src=(0, 0, 0, 0)) -> np.ndarray:
    """Meson::contract + fourier(FORWARD): [Lt, Nmom, 2]."""
    n = len(momenta(Q_sq))
    out = np.zeros((L[3], n, 2))
    lib().orc_meson_2pt(_L(L), _ptr(np.ascontiguousarray(prop)), op, Q_sq, _L(x_src), _ptr(out))
    return out


def baryon_2pt(L, prop1, prop2, op, Q_sq=0, x_src=(0, 0, 0, 0)) -> np.ndarray:
    """Baryon::contract + fourier(FORWARD): [Lt, Nmom, 4, 4, 2]."""
    n = len(momenta(Q_sq))
    out = np.zeros((L[3], n, 4, 4, 2))
    lib().orc_baryon_2pt(_L(L), _ptr(np.ascontiguousarray(prop1)), _ptr(np.ascontiguousarray(prop2)), op, Q_sq,
                         _L(x_src), _ptr(out))
    return out


DELTAS = ["ISO1", "ISO1O2"]


def delta_2pt(L, prop1, prop2, op, Q_sq=0, x_src=(0, 0, 0, 0)) -> np.ndarray:
    """Baryon_Dec::contract + fourier(FORWARD): [Lt, Nmom, 3, 4, 4, 2]."""
    n = len(momenta(Q_sq))
    out = np.zeros((L[3], n, 3, 4, 4, 2))
    lib().orc_delta_2pt(_L(L), _ptr(np.ascontiguousarray(prop1)), _ptr(np.ascontiguousarray(prop2)), op, Q_sq,
                        _L(x_src), _ptr(out))
    return out


def nucleon_2pt(L, prop1, prop2, Q_sq=0, x_src=(0, 0, 0, 0)) -> np.ndarray:
    """contractNucleon (lib/lattice_util.cpp:3374): [Lt, Nmom, 4, 4, 2]."""
    n = len(momenta(Q_sq))
    out = np.zeros((L[3], n, 4, 4, 2))
    lib().orc_nucleon_2pt(_L(L), _ptr(np.ascontiguousarray(prop1)), _ptr(np.ascontiguousarray(prop2)), Q_sq,
                          _L(x_src), _ptr(out))
    return out


def ref_delta_2pt(L, prop1, prop2, op, Q_sq=0, x_src=(0, 0, 0, 0)) -> np.ndarray:
    n = len(momenta(Q_sq))
    out = np.zeros((L[3], n, 3, 4, 4, 2))
    ref().ref_delta_2pt(_L(L), _ptr(np.ascontiguousarray(prop1)), _ptr(np.ascontiguousarray(prop2)), op, Q_sq,
                        _L(x_src), _ptr(out))
    return out


def ref_contract_nucleon_text(L, prop1, prop2, Q_sq, x_src, path) -> np.ndarray:
    """contractNucleon of the compiled reference: it writes its correlator as text to
    `path`; returned as [Lt, Nmom, 4, 4, 2] at the printed precision (%+e, 7 digits)."""
    ref().ref_contract_nucleon(_L(L), _ptr(np.ascontiguousarray(prop1)), _ptr(np.ascontiguousarray(prop2)), Q_sq,
                               _L(x_src), os.fsencode(str(path)))
    rows = [ln.split() for ln in open(path) if ln.strip()]
    n = len(momenta(Q_sq))
    return np.array([[float(r[-2]), float(r[-1])] for r in rows]).reshape(L[3], n, 4, 4, 2)


def ref_meson_2pt(L, prop, op, Q_sq=0, x_src=(0, 0, 0, 0)) -> np.ndarray:
    n = len(momenta(Q_sq))
    out = np.zeros((L[3], n, 2))
    ref().ref_meson_2pt(_L(L), _ptr(np.ascontiguousarray(prop)), op, Q_sq, _L(x_src), _ptr(out))
    return out


def ref_baryon_2pt(L, prop1, prop2, op, Q_sq=0, x_src=(0, 0, 0, 0)) -> np.ndarray:
    n = len(momenta(Q_sq))
    out = np.zeros((L[3], n, 4, 4, 2))
    ref().ref_baryon_2pt(_L(L), _ptr(np.ascontiguousarray(prop1)), _ptr(np.ascontiguousarray(prop2)), op, Q_sq,
                         _L(x_src), _ptr(out))
    return out
