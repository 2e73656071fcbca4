"""Generate the golden vectors in tests/golden/ from the REFERENCE itself.

The reference's hot-path sources are compiled unmodified (oracle/ref/Makefile)
into oracle/_ref/libqkxref.so; this script runs the reference's own
Vector::tm / tm_xx / chiral / BLAS / CG::operator() on seeded synthetic inputs
and stores the outputs.  The inputs are NOT stored: they are regenerated by
the oracle's counter-based generator from the seeds recorded here, and a
checksum of the inputs is stored so that a change of the generator is caught.

    python tests/golden/make_golden.py          (needs the reference sources)

Fixtures:
  ref_ops_small.npz   full outputs of every operator, lattice 4x2x2x4
  ref_ops_probe.npz   per operator: |out|^2 and <w_k, out> for 3 fixed probe
                      fields w_k, plus the full output on 16 sampled sites,
                      lattice 4x4x4x8
  ref_cg.npz          CG::operator() solution probes and true residual,
                      lattices 4x4x4x8 and 8x8x8x16
  ref_smear.npz       Gauge::calculatePlaquette, qcd_projectSU33d, Gauge::APE_smearing,
                      Vector::Gaussian_smearing and the propagator loop of
                      bin/test_invert_prop.cpp, lattice 4x4x4x8

  ref_contract.npz    Meson::contract / Baryon::contract / Baryon_Dec::contract +
                      fourier(FORWARD) on seeded propagators, lattice 4x2x4x4, and
                      the numbers contractNucleon prints for them (its text output)
  ref_conf_4x2x2x4.lime
                      an ILDG configuration written by the reference's own
                      qkxTM_writeGaugeLime (lib/write_conf_lime.cpp, compiled with
                      the LIME and MPI-IO stand-ins of oracle/ref), links
                      apply_bc(gauge_random(L, 0.3, LIME_SEED)), message LIME_MESSAGE

    python tests/golden/make_golden.py smear      (only ref_smear.npz)
    python tests/golden/make_golden.py contract   (only ref_contract.npz)
    python tests/golden/make_golden.py lime       (only ref_conf_4x2x2x4.lime)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

KAPPA, MU = 0.16, 0.01
EPS = 0.3
# operators also stored with twistSign = -1
TWIST_SIGN_OPS = ["tm", "tm_dag", "twist_inv", "tm_xx_ee", "tm_xx_dagtm_xx_oo", "tm_xx_chiral_oo",
                  "tm_xx_dagtm_xx_chiral_ee"]


def inputs(L, seed_u, seed_psi, bc=True):
    U = O.gauge_random(L, EPS, seed_u)
    if bc:
        U = O.apply_bc(L, U, -1)
    psi = O.spinor_gaussian(L, seed_psi)
    return U, psi


def checksum(a: np.ndarray) -> np.ndarray:
    w = np.linspace(0.5, 1.5, a.size).reshape(a.shape)
    return np.array([a.sum(), (a * w).sum(), (a * a).sum()])


def probes(L, n=3, seed=9000):
    return [O.spinor_gaussian(L, seed + k) for k in range(n)]


def sample_sites(L, n=16):
    V = O.volume(L)
    return np.unique(np.linspace(0, V - 1, n).astype(np.int64))


def perturbed_links(L, U, scale, seed):
    """U plus scale times unit normals (three Gaussian spinor fields fill the 72 reals of a site)."""
    g = np.concatenate([O.spinor_gaussian(L, seed + k).reshape(-1, 24) for k in range(3)], axis=1)
    return U + scale * g.reshape(U.shape)


SMEAR = {"L": (4, 4, 4, 8), "seed_u": 51, "seed_psi": 52, "seed_pert": 53, "ape_n": 20, "ape_alpha": 0.5,
         "gauss_n": 50, "gauss_alpha": 4.0, "prop_n": 5, "prop_alpha": 4.0, "prop_src": (1, 2, 3, 5),
         "prop_tol": 1e-12}


def make_smear():
    c = SMEAR
    L = c["L"]
    U = O.gauge_random(L, EPS, c["seed_u"])
    psi = O.spinor_gaussian(L, c["seed_psi"])
    sites = sample_sites(L)
    W = probes(L)
    d = {k: np.array(v) for k, v in c.items()}
    d["eps"], d["kappa"], d["mu"] = EPS, KAPPA, MU
    d["sites"] = sites
    d["in_checksum"] = np.concatenate([checksum(U), checksum(psi)])
    Ubc = O.apply_bc(L, U, -1)
    d["plaq"] = np.array([O.ref_plaquette(L, U)])
    d["plaq_bc"] = np.array([O.ref_plaquette(L, Ubc)])
    P = O.ref_project_su3(L, perturbed_links(L, U, 0.3, c["seed_pert"]))
    d["proj:sites"] = P[sites]
    d["proj:checksum"] = checksum(P)
    for n in (1, 2):
        A = O.ref_ape_smear(L, U, n, c["ape_alpha"])
        d[f"ape{n}:sites"] = A[sites]
        d[f"ape{n}:checksum"] = checksum(A)
    A = O.ref_ape_smear(L, U, c["ape_n"], c["ape_alpha"])
    d["ape:sites"] = A[sites]
    d["ape:checksum"] = checksum(A)
    d["ape:plaq"] = np.array([O.ref_plaquette(L, A)])
    for n in (1, c["gauss_n"]):
        g = O.ref_gaussian_smear(L, A, psi, n, c["gauss_alpha"])
        d[f"gauss{n}:sites"] = g[sites]
        d[f"gauss{n}:norm2"] = np.array([np.sum(g * g)])
        d[f"gauss{n}:probe"] = np.array([np.sum(w * g) for w in W])
    src = c["prop_src"]
    s = src[0] + L[0] * (src[1] + L[1] * (src[2] + L[2] * src[3]))
    prop = O.ref_propagator(L, Ubc, A, KAPPA, MU, c["prop_n"], c["prop_alpha"], src=s, tol=c["prop_tol"],
                            maxIter=2000)
    d["prop:sites"] = prop[sites]
    d["prop:norm2"] = np.array([np.sum(prop * prop)])
    d["prop:checksum"] = checksum(prop)
    np.savez_compressed(os.path.join(HERE, "ref_smear.npz"), **d)
    print("ref_smear.npz", os.path.getsize(os.path.join(HERE, "ref_smear.npz")), "bytes")


def seeded_propagator(L, seed):
    """[V, 4, 4, 3, 3, 2] from 12 Gaussian spinor fields of the oracle's generator."""
    f = np.stack([O.spinor_gaussian(L, seed + k) for k in range(12)], axis=1)  # [V, 12, 4, 3, 2]
    return np.ascontiguousarray(f.reshape(-1, 4, 3, 4, 3, 2).transpose(0, 3, 1, 4, 2, 5))


CONTRACT = {"L": (4, 2, 4, 4), "seed1": 61, "seed2": 81, "Q_sq": 2, "x_src": (1, 0, 3, 2)}


def make_contract():
    c = CONTRACT
    L = c["L"]
    p1, p2 = seeded_propagator(L, c["seed1"]), seeded_propagator(L, c["seed2"])
    d = {k: np.array(v) for k, v in c.items()}
    d["in_checksum"] = np.concatenate([checksum(p1), checksum(p2)])
    d["momenta"] = O.momenta(c["Q_sq"])
    for op, name in enumerate(O.MESONS):
        d[f"meson:{name}"] = O.ref_meson_2pt(L, p1, op, c["Q_sq"], c["x_src"])
    for op, name in enumerate(O.BARYONS):
        d[f"baryon:{name}"] = O.ref_baryon_2pt(L, p1, p2, op, c["Q_sq"], c["x_src"])
    for op, name in enumerate(O.DELTAS):
        d[f"delta:{name}"] = O.ref_delta_2pt(L, p1, p2, op, c["Q_sq"], c["x_src"])
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        d["nucleon_text"] = O.ref_contract_nucleon_text(L, p1, p2, c["Q_sq"], c["x_src"], os.path.join(tmp, "n.txt"))
    np.savez_compressed(os.path.join(HERE, "ref_contract.npz"), **d)
    print("ref_contract.npz", os.path.getsize(os.path.join(HERE, "ref_contract.npz")), "bytes")


LIME_L = (4, 2, 2, 4)
LIME_SEED = 77
LIME_MESSAGE = b"written by the reference's qkxTM_writeGaugeLime"


def make_lime():
    U = O.apply_bc(LIME_L, O.gauge_random(LIME_L, EPS, LIME_SEED), -1)
    path = os.path.join(HERE, "ref_conf_4x2x2x4.lime")
    O.ref_write_gauge_lime(path, LIME_L, U, LIME_MESSAGE)
    print(os.path.basename(path), os.path.getsize(path), "bytes")


def main():
    O.build(ref=True)
    if not O.ref_available():
        raise SystemExit("reference build missing (oracle/_ref/libqkxref.so)")
    if sys.argv[1:] == ["smear"]:
        make_smear()
        return
    if sys.argv[1:] == ["contract"]:
        make_contract()
        return
    if sys.argv[1:] == ["lime"]:
        make_lime()
        return

    # --- small lattice, full outputs
    L = (4, 2, 2, 4)
    U, psi = inputs(L, 11, 12)
    d = {"L": np.array(L), "kappa": KAPPA, "mu": MU, "eps": EPS, "seed_u": 11, "seed_psi": 12,
         "bc": 1, "in_checksum": np.concatenate([checksum(U), checksum(psi)])}
    for op in O.REF_OPS:
        d[f"{op}@1"] = O.ref_apply(op, L, U, psi, KAPPA, MU, 1)
    for op in TWIST_SIGN_OPS:
        d[f"{op}@-1"] = O.ref_apply(op, L, U, psi, KAPPA, MU, -1)
    np.savez_compressed(os.path.join(HERE, "ref_ops_small.npz"), **d)

    # --- 4^3x8, probes
    L = (4, 4, 4, 8)
    U, psi = inputs(L, 21, 22)
    W = probes(L)
    sites = sample_sites(L)
    d = {"L": np.array(L), "kappa": KAPPA, "mu": MU, "eps": EPS, "seed_u": 21, "seed_psi": 22,
         "bc": 1, "probe_seed": 9000, "sites": sites,
         "in_checksum": np.concatenate([checksum(U), checksum(psi)])}
    for op in O.REF_OPS:
        out = O.ref_apply(op, L, U, psi, KAPPA, MU, 1)
        d[f"{op}:norm2"] = np.array([np.sum(out * out)])
        d[f"{op}:probe"] = np.array([np.sum(w * out) for w in W])
        d[f"{op}:sites"] = out[sites]
    # BLAS of the reference
    x = psi.copy()
    y = O.spinor_gaussian(L, 23)
    d["blas:redot"] = np.array([O.ref().ref_blas(0, O._L(L), 0.0, O._ptr(x.copy()), O._ptr(y))])
    x1 = x.copy()
    O.ref().ref_blas(1, O._L(L), 0.37, O._ptr(x1), O._ptr(y))
    d["blas:axpy:sites"] = x1[sites]
    x2 = x.copy()
    O.ref().ref_blas(2, O._L(L), -0.41, O._ptr(x2), O._ptr(y))
    d["blas:xpay:sites"] = x2[sites]
    d["blas:norm2"] = np.array([O.ref().ref_blas(3, O._L(L), 0.0, O._ptr(x.copy()), O._ptr(y))])
    np.savez_compressed(os.path.join(HERE, "ref_ops_probe.npz"), **d)

    # --- CG::operator() (lib/solvers.cpp) as bin/test_invert.cpp drives it:
    # in = M^+ b, links with the antiperiodic boundary applied, x zero.
    d = {}
    for tag, L, seed_u, seed_b in (("4x4x4x8", (4, 4, 4, 8), 31, 32), ("8x8x8x16", (8, 8, 8, 16), 41, 42)):
        U, b = inputs(L, seed_u, seed_b)
        Mdb = O.ref_apply("tm_dag", L, U, b, KAPPA, MU, 1)
        xr = O.ref_cg(L, U, Mdb, KAPPA, MU, 1, tol=1e-10, maxIter=1000)
        W = probes(L)
        res = b - O.ref_apply("tm", L, U, xr, KAPPA, MU, 1)
        d[f"{tag}:L"] = np.array(L)
        d[f"{tag}:seeds"] = np.array([seed_u, seed_b])
        d[f"{tag}:x_norm2"] = np.array([np.sum(xr * xr)])
        d[f"{tag}:x_probe"] = np.array([np.sum(w * xr) for w in W])
        d[f"{tag}:x_sites"] = xr[sample_sites(L)]
        d[f"{tag}:true_residual"] = np.array([np.sqrt(np.sum(res * res) / np.sum(b * b))])
        _, iters, trace = O.cg(L, U, Mdb, KAPPA, MU, 1, tol=1e-10, maxIter=1000)
        d[f"{tag}:iters_oracle"] = np.array([iters])
        d[f"{tag}:r2_trace_oracle"] = trace
        d[f"{tag}:in_checksum"] = np.concatenate([checksum(U), checksum(b)])
    d["kappa"], d["mu"], d["eps"] = KAPPA, MU, EPS
    np.savez_compressed(os.path.join(HERE, "ref_cg.npz"), **d)
    for f in ("ref_ops_small.npz", "ref_ops_probe.npz", "ref_cg.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
    make_smear()
    make_contract()
    make_lime()


if __name__ == "__main__":
    main()
