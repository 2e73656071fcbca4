"""CPU tests of the learned preconditioner's oracle (oracle/qkx_oracle_ptc.c): the
gradient against finite differences, linearity, gauge covariance and the
identity initialisation.  The network has no reference counterpart; these
properties pin the restatement that the GPU kernels are checked against."""
import numpy as np

L = (4, 2, 2, 4)
CH = [4, 3, 2, 4]


def _setup(O, seed=5):
    U = O.apply_bc(L, O.gauge_random(L, 0.3, seed), -1)
    n = O.ptc_nweights(CH)
    W = np.random.default_rng(seed).standard_normal((n, 2)) * 0.3
    return U, W


def test_gradient_matches_finite_differences(oracle):
    U, W = _setup(oracle)
    r = oracle.spinor_gaussian(L, 1)
    e = oracle.spinor_gaussian(L, 2)
    _, g = oracle.ptc_loss_grad(L, U, CH, W, r, e)
    h = 1e-6
    rng = np.random.default_rng(3)
    for k in rng.choice(W.shape[0], 16, replace=False):
        for part in (0, 1):
            Wp, Wm = W.copy(), W.copy()
            Wp[k, part] += h
            Wm[k, part] -= h
            fd = (oracle.ptc_loss_grad(L, U, CH, Wp, r, e, False)[0] -
                  oracle.ptc_loss_grad(L, U, CH, Wm, r, e, False)[0]) / (2 * h)
            # dL/dRe W = 2 Re(dL/dW*), dL/dIm W = 2 Im(dL/dW*)
            assert abs(fd - 2 * g[k, part]) <= 1e-6 * max(1.0, abs(fd)), (k, part, fd, 2 * g[k, part])


def test_linearity(oracle):
    U, W = _setup(oracle)
    a, b = oracle.spinor_gaussian(L, 3), oracle.spinor_gaussian(L, 4)
    na, nb = oracle.ptc_forward(L, U, CH, W, a), oracle.ptc_forward(L, U, CH, W, b)
    nab = oracle.ptc_forward(L, U, CH, W, 0.7 * a - 1.3 * b)
    assert np.abs(nab - (0.7 * na - 1.3 * nb)).max() < 1e-12 * np.abs(nab).max()


def _cx(a):
    return a[..., 0] + 1j * a[..., 1]


def _re(z):
    return np.stack([z.real, z.imag], -1)


def test_gauge_covariance(oracle):
    """N[U^g](g r) = g N[U](r) with U^g_mu(x) = g(x) U_mu(x) g(x+mu)^+."""
    U, W = _setup(oracle)
    G = _cx(oracle.gauge_random(L, 1.0, 99))[:, 0]  # one SU(3) matrix per site
    Uc = _cx(U)
    V = Uc.shape[0]

    def nbr(s, mu):
        c = [s % L[0], (s // L[0]) % L[1], (s // (L[0] * L[1])) % L[2], s // (L[0] * L[1] * L[2])]
        c[mu] = (c[mu] + 1) % L[mu]
        return c[0] + L[0] * (c[1] + L[1] * (c[2] + L[2] * c[3]))

    Ug = np.empty_like(Uc)
    for s in range(V):
        for mu in range(4):
            Ug[s, mu] = G[s] @ Uc[s, mu] @ G[nbr(s, mu)].conj().T
    r = _cx(oracle.spinor_gaussian(L, 7))
    rg = np.einsum("xab,xsb->xsa", G, r)
    out = _cx(oracle.ptc_forward(L, _re(Uc), CH, W, _re(r)))
    outg = _cx(oracle.ptc_forward(L, _re(Ug), CH, W, _re(rg)))
    assert np.abs(outg - np.einsum("xab,xsb->xsa", G, out)).max() < 1e-12 * np.abs(out).max()


def test_identity_path_only_is_identity(oracle):
    U, _ = _setup(oracle)
    ch = [4, 8, 4]
    W = np.zeros((oracle.ptc_nweights(ch), 2))
    # layer 0: 4 -> 8, identity path copies spin a to channel a; layer 1: 8 -> 4 takes it back
    for a in range(4):
        W[a * 4 + a, 0] = 1.0
    off = 9 * 8 * 4
    for a in range(4):
        W[off + a * 8 + a, 0] = 1.0
    r = oracle.spinor_gaussian(L, 8)
    assert np.array_equal(oracle.ptc_forward(L, U, ch, W, r), r)


def test_bf16_activation_mode(oracle):
    """The BF16 mode rounds the hidden activations (and only those): the output moves by
    about a BF16 rounding (2^-9 relative), its hidden inputs are exactly representable in
    BF16, and a one-layer network (no hidden activation) is unchanged."""
    U, W = _setup(oracle)
    r = oracle.spinor_gaussian(L, 8)
    a = oracle.ptc_forward(L, U, CH, W, r)
    b = oracle.ptc_forward(L, U, CH, W, r, bf16=True)
    d = np.linalg.norm(a - b) / np.linalg.norm(a)
    assert 0 < d < 2.0 ** -7
    one = [4, 4]
    W1 = W[:oracle.ptc_nweights(one)]
    assert np.array_equal(oracle.ptc_forward(L, U, one, W1, r), oracle.ptc_forward(L, U, one, W1, r, bf16=True))
    # the mode is reset after each call
    assert np.array_equal(oracle.ptc_forward(L, U, CH, W, r), a)
    # widths 4 -> 4 -> 4 with an identity first layer: the hidden activation is r rounded to BF16
    ident = np.zeros((oracle.ptc_nweights([4, 4, 4]), 2))
    for c in range(4):
        ident[c * 4 + c, 0] = 1.0                  # layer 0, path 0
        ident[9 * 16 + c * 4 + c, 0] = 1.0         # layer 1, path 0
    y = oracle.ptc_forward(L, U, [4, 4, 4], ident, r, bf16=True)
    bits = y.astype(np.float32).view(np.uint32)
    assert np.all(bits & 0xFFFF == 0)
    assert np.abs(y - r).max() <= 2.0 ** -8 * np.abs(r).max()
