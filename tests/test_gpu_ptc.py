"""GPU tests of the learned preconditioner (no reference counterpart): the forward
and backward kernels against the CPU oracle at the same BF16-rounded weights,
training on the library's own solves, and the batched even-odd flexible CG that
uses it (true residual checked in FP64 by the oracle, iterations against the
same solver without the network, and the plain-solver fallback).

Tolerances.  The kernels store the hidden activations and the activation
gradients between layers in BF16 and compute in FP32 (BF16 weights, FP32 tile
sums, FP64 across tiles).  Against the oracle in its BF16-activation mode (the
same roundings, FP64 arithmetic) the only differences are FP32 arithmetic and
the rare BF16 rounding it flips, amplified by the later layers: forward 1e-3
relative, loss 2e-3, gradient 2e-3 (norm-relative).  Against the plain FP64 oracle the BF16 storage itself
shows (2^-9 a rounding): 2e-2.  The tensor-core layer also rounds the
transported activations to BF16 before the MMA: 2e-2 against both."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

L = (4, 4, 4, 8)
KAPPA, MU = 0.16, 0.01
CH = (4, 16, 16, 16, 4)


@pytest.fixture(scope="module")
def setup(qkx, oracle):
    U = oracle.apply_bc(L, oracle.gauge_random(L, 0.3, 2024), -1)
    lat = qkx.Lattice(qkx.LatticeInfo(L=L, kappa=KAPPA, mu=MU))
    lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
    yield lat, U
    lat.close()


def U_of(setup):
    return setup[1]


@pytest.mark.parametrize("ch", [CH, (4, 8, 4), (4, 16, 8, 4), (4, 16, 16, 4), (4, 4, 4)])
def test_forward_matches_oracle(qkx, oracle, setup, ch):
    lat, U = setup
    net = qkx.Ptc(lat, ch, seed=11, init_scale=0.3, tensor_cores=False)
    W = net.weights(1)
    for seed in (1, 2):
        r = oracle.spinor_gaussian(L, seed)
        got = net.apply(r)
        exp = oracle.ptc_forward(L, U, list(ch), W, r, bf16=True)
        assert rel(got, exp) < 1e-3, (ch, rel(got, exp))
        assert rel(got, oracle.ptc_forward(L, U, list(ch), W, r)) < 2e-2
    net.close()


@pytest.mark.parametrize("Lt", [(4, 4, 4, 8), (6, 4, 2, 10), (8, 8, 8, 16)])
def test_tensor_core_layer(qkx, oracle, Lt):
    """tcgen05 16 -> 16 layers (BF16 activations) against the FP32 kernels and the oracle,
    including a lattice whose half volume is not a multiple of the 128-site tile."""
    U = oracle.apply_bc(Lt, oracle.gauge_random(Lt, 0.3, 31), -1)
    with qkx.Lattice(qkx.LatticeInfo(L=Lt, kappa=KAPPA, mu=MU)) as lat:
        lat.load_gauge(U, qkx.LINKS_AS_GIVEN)
        ref = qkx.Ptc(lat, CH, seed=12, init_scale=0.3, tensor_cores=False)
        tc = qkx.Ptc(lat, CH, seed=99, init_scale=0.3, tensor_cores=True)
        tc.set_weights(ref.weights(0))
        r = oracle.spinor_gaussian(Lt, 6)
        a, b = ref.apply(r), tc.apply(r)
        assert rel(b, a) < 2e-2, rel(b, a)
        assert rel(b, oracle.ptc_forward(Lt, U, list(CH), ref.weights(1), r, bf16=True)) < 2e-2
        assert rel(a, oracle.ptc_forward(Lt, U, list(CH), ref.weights(1), r, bf16=True)) < 1e-3
        ref.close()
        tc.close()


def test_identity_at_zero_init(qkx, oracle, setup):
    lat, _ = setup
    net = qkx.Ptc(lat, CH, seed=1, init_scale=0.0, tensor_cores=False)
    r = oracle.spinor_gaussian(L, 3)
    # the identity network returns r through BF16 hidden activations: r rounded to BF16
    y = net.apply(r)
    assert rel(y, r) < 2.0 ** -8
    assert np.array_equal(y, oracle.ptc_forward(L, U_of(setup), list(CH), net.weights(1), r, bf16=True))
    net.close()


@pytest.mark.parametrize("tc", [False, True])
def test_loss_and_gradient_match_oracle(qkx, oracle, setup, tc):
    """FP32-pipe layers to 2e-3; the tensor-core layers (transport in BF16, BF16 MMA
    operands) to 2e-2."""
    lat, U = setup
    tol = 2e-2 if tc else 2e-3
    for ch in (CH, (4, 8, 4)):
        net = qkx.Ptc(lat, ch, seed=5, init_scale=0.3, tensor_cores=tc)
        W = net.weights(1)
        r = oracle.spinor_gaussian(L, 4)
        e = oracle.spinor_gaussian(L, 5)
        loss, g = net.loss_grad(r, e)
        lo, go = oracle.ptc_loss_grad(L, U, list(ch), W, r, e, bf16=True)
        assert abs(loss - lo) < tol * lo
        assert rel(g, go) < tol, (ch, tc, rel(g, go))
        # fixed-order reductions: the same gradient twice
        loss2, g2 = net.loss_grad(r, e)
        assert loss2 == loss and np.array_equal(g, g2)
        net.close()


@pytest.fixture(scope="module")
def trained(qkx, setup):
    lat, _ = setup
    net = qkx.Ptc(lat, CH, seed=3, init_scale=0.05)
    info = net.train(n_solves=16, steps=400, lr=3e-3, solve_tol=1e-7, seed=9)
    yield net, info
    net.close()


def test_training_reduces_loss(trained):
    _, info = trained
    assert info["steps"] == 400
    assert info["loss_final"] < 0.5 * info["loss_initial"], info


def test_gcr_with_learned_preconditioner(qkx, oracle, setup, trained):
    lat, U = setup
    net, _ = trained
    bs = [oracle.spinor_gaussian(L, 40 + k) for k in range(3)]
    xs, info = lat.invert(bs, method=qkx.SOLVER_GCR_PTC, tol=1e-10, preconditioner=net)
    assert info.converged == 1 and info.fallbacks == 0
    for b, x in zip(bs, xs):
        r = b - oracle.apply("tm", L, U, x, KAPPA, MU)
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10
    _, plain = lat.invert(bs, method=qkx.SOLVER_GCR_PTC, tol=1e-10, preconditioner=None)
    assert plain.converged == 1
    # what the trained network gains or loses against the same solver without it: on this
    # well-conditioned system the unpreconditioned normal equations take ~40 iterations and a
    # three-hop network does not shorten that (it may lengthen it); the preconditioned solve
    # must stay within twice the plain count
    print(f"learned: {info.iterations} iterations, {info.restarts} passes; "
          f"without the network: {plain.iterations}, {plain.restarts}")
    assert info.iterations <= 2 * plain.iterations, (info.iterations, plain.iterations)
    # an identity network (zero hop weights) is the unpreconditioned solver up to BF16 rounding
    ident = qkx.Ptc(lat, CH, seed=1, init_scale=0.0, tensor_cores=False)
    try:
        _, same = lat.invert(bs, method=qkx.SOLVER_GCR_PTC, tol=1e-10, preconditioner=ident)
        assert same.converged == 1 and abs(same.iterations - plain.iterations) <= 2, (same.iterations,
                                                                                        plain.iterations)
    finally:
        ident.close()


def test_six_layer_network_cuts_the_iterations(qkx, oracle, setup):
    """The gain the learned part is for: a six-layer network (reach six hops) trained on this
    configuration's Schur pairs shortens the flexible CG against the same solver without it,
    each solution to 1e-10 by the oracle."""
    lat, U = setup
    net = qkx.Ptc(lat, (4, 16, 16, 16, 16, 16, 4), seed=3, init_scale=0.05)
    try:
        info_t = net.train(n_solves=16, steps=400, lr=3e-3, solve_tol=1e-7, seed=9)
        assert info_t["loss_final"] < 0.2 * info_t["loss_initial"], info_t
        bs = [oracle.spinor_gaussian(L, 60 + k) for k in range(3)]
        xs, info = lat.invert(bs, method=qkx.SOLVER_GCR_PTC, tol=1e-10, preconditioner=net)
        _, plain = lat.invert(bs, method=qkx.SOLVER_GCR_PTC, tol=1e-10, preconditioner=None)
        print(f"six layers: {info.iterations} iterations against {plain.iterations} without the network")
        assert info.converged == 1 and info.fallbacks == 0
        assert info.iterations < plain.iterations, (info.iterations, plain.iterations)
        for b, x in zip(bs, xs):
            r = b - oracle.apply("tm", L, U, x, KAPPA, MU)
            assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10
    finally:
        net.close()


def test_gcr_fallback_to_plain_solver(qkx, oracle, setup):
    lat, U = setup
    b = oracle.spinor_gaussian(L, 77)
    (x,), info = lat.invert([b], method=qkx.SOLVER_GCR_PTC, tol=1e-10, maxIter=2, preconditioner=None)
    assert info.fallbacks == 1 and info.converged == 1
    r = b - oracle.apply("tm", L, U, x, KAPPA, MU)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10


def test_ptc_argument_checks(qkx, setup):
    lat, _ = setup
    with pytest.raises(qkx.QkxError) as e:
        qkx.Ptc(lat, (4, 12, 4))
    assert e.value.code == qkx.ERR_INVALID
    with pytest.raises(qkx.QkxError) as e:
        qkx.Ptc(lat, (8, 16, 4))
    assert e.value.code == qkx.ERR_INVALID


def test_learned_solver_per_rhs_masses_and_zero_source(qkx, oracle, setup):
    """The batched learned solver takes a twisted mass per right-hand side (qkx_solver_params.mu)
    and returns x = 0 for a zero source, the others to 1e-10 by the oracle."""
    import ctypes as C
    lat, U = setup
    mus = [0.004, 0.01, 0.02]
    bs = [oracle.spinor_gaussian(L, 80), np.zeros((oracle.volume(L), 4, 3, 2)), oracle.spinor_gaussian(L, 81)]
    xs = [np.empty_like(b) for b in bs]
    n = len(bs)
    arr = (C.c_double * n)(*mus)
    sp = qkx.SolverParams(qkx.SOLVER_GCR_PTC, qkx.PREC_HALF, 1e-10, 10000, 0.0, 1,
                          C.cast(arr, C.POINTER(C.c_double)), None)
    info = qkx.SolveInfo()
    bp = (C.c_void_p * n)(*[b.ctypes.data for b in bs])
    xp = (C.c_void_p * n)(*[x.ctypes.data for x in xs])
    qkx.check(qkx.lib().qkx_invert(lat.ctx, C.byref(sp), n, bp, xp, C.byref(info)))
    assert info.converged == 1
    assert not xs[1].any()
    for mu, b, x in ((mus[0], bs[0], xs[0]), (mus[2], bs[2], xs[2])):
        r = b - oracle.apply("tm", L, U, x, KAPPA, mu)
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10
