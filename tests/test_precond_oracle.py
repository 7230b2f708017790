"""CPU checks of the learned-preconditioner oracle: analytic gradients against central finite
differences, the probe hash, the algebra of the factorised preconditioner, and the gauge basis."""
import numpy as np
import pytest

from oracle import precond_gnn as og
from precond_cases import reduced_blocks, small_sequence


@pytest.fixture(scope="module")
def system():
    N, bi, bl, bs, diag, S = reduced_blocks(small_sequence(), 1e-6)
    g = og.Graph(N, bi, bl)
    xe, xn, cinv = og.features(g, bs, diag)
    return g, xe, xn, cinv, S


def random_weights(seed, out_scale=0.05):
    rng = np.random.default_rng(seed)
    w = np.zeros(og.NWEIGHTS)
    for name, (o, k, n) in og.LAYOUT.items():
        s = out_scale if name == "out" else 1.0 / np.sqrt(k)
        w[o:o + (k + 1) * n] = rng.uniform(-s, s, size=(k + 1) * n)
    return w


def dense_factor(g, xe, coef):
    n = 6 * g.N
    I_E = np.eye(n)
    E = og.edge_blocks(xe, coef)
    F = np.zeros((n, n))
    for k in range(g.ne):
        a, b = g.ea[k], g.eb[k]
        I_E[6 * b:6 * b + 6, 6 * a:6 * a + 6] += E[k]
        F[6 * b:6 * b + 6, 6 * a:6 * a + 6] = xe[k, :36].reshape(6, 6)
    return I_E, np.eye(n) + F + F.T


def test_layout_size():
    assert og.NWEIGHTS == 61059


def test_probe_hash_matches_integer_restatement():
    def fmix(idx, seed):
        h = (idx * 0x9E3779B1 + seed) & 0xFFFFFFFF
        h ^= h >> 16
        h = (h * 0x85EBCA6B) & 0xFFFFFFFF
        h ^= h >> 13
        h = (h * 0xC2B2AE35) & 0xFFFFFFFF
        h ^= h >> 16
        return 1.0 if h & 1 else -1.0
    z = og.probe_signs(12345, 500)
    assert np.array_equal(z, [fmix(i, 12345) for i in range(500)])
    assert abs(z.mean()) < 0.2


def test_normalised_blocks_reproduce_the_system(system):
    g, xe, xn, cinv, S = system
    Cinv = np.zeros_like(S)
    for i in range(g.N):
        Cinv[6 * i:6 * i + 6, 6 * i:6 * i + 6] = cinv[i]
    Sh = Cinv @ S @ Cinv.T
    assert np.allclose(np.diagonal(Sh), 1.0)
    for k in range(g.ne):
        a, b = g.ea[k], g.eb[k]
        assert np.allclose(Sh[6 * b:6 * b + 6, 6 * a:6 * a + 6], xe[k, :36].reshape(6, 6), atol=1e-12)


def test_probe_loss_equals_dense_formula(system):
    g, xe, xn, cinv, S = system
    rng = np.random.default_rng(1)
    coef = rng.normal(scale=0.2, size=(g.ne, 3))
    loss, _ = og.probe_loss(g, xe, coef, 7)
    n = 6 * g.N
    I_E, Sh = dense_factor(g, xe, coef)
    P = I_E @ Sh @ I_E.T
    Z = og.probe_signs(7, n * og.PROBES).reshape(n, og.PROBES)
    dense = ((P @ Z - Z) ** 2).sum() / (n * og.PROBES)
    assert loss == pytest.approx(dense, rel=1e-12)


def test_dcoef_matches_finite_differences(system):
    g, xe, xn, cinv, S = system
    rng = np.random.default_rng(2)
    coef = rng.normal(scale=0.2, size=(g.ne, 3))
    _, dcoef = og.probe_loss(g, xe, coef, 11)
    h = 1e-6
    for k, c in [(0, 0), (g.ne // 2, 1), (g.ne - 1, 2)]:
        cp, cm = coef.copy(), coef.copy()
        cp[k, c] += h
        cm[k, c] -= h
        fd = (og.probe_loss(g, xe, cp, 11)[0] - og.probe_loss(g, xe, cm, 11)[0]) / (2 * h)
        assert dcoef[k, c] == pytest.approx(fd, rel=1e-5, abs=1e-10)


def test_weight_gradient_matches_finite_differences(system):
    g, xe, xn, cinv, S = system
    w = random_weights(3)
    loss, grad, _ = og.loss_and_grad(w, g, xe, xn, 5)
    rng = np.random.default_rng(4)
    h = 1e-6
    for name, (o, k, n) in og.LAYOUT.items():
        for idx in rng.integers(o, o + (k + 1) * n, size=3):
            wp, wm = w.copy(), w.copy()
            wp[idx] += h
            wm[idx] -= h
            fd = (og.loss_and_grad(wp, g, xe, xn, 5)[0] - og.loss_and_grad(wm, g, xe, xn, 5)[0]) / (2 * h)
            assert grad[idx] == pytest.approx(fd, rel=1e-4, abs=1e-9), (name, idx)


def test_unit_coefficients_improve_conditioning(system):
    """c = 1 (an untrained network) is the first-order FSAI factor: the preconditioned spectrum
    is tighter than block-Jacobi's."""
    g, xe, xn, cinv, S = system
    I_E, Sh = dense_factor(g, xe, np.zeros((g.ne, 3)))
    ev_j = np.linalg.eigvalsh(Sh)
    ev_l = np.linalg.eigvalsh(I_E @ Sh @ I_E.T)
    assert ev_l[-1] / ev_l[0] < ev_j[-1] / ev_j[0]


def test_gauge_basis_spans_the_near_null_space():
    """S Z = O(lambda): the camera parts of the 7 similarity motions are the near-null space of
    the damped reduced system, at any parameters."""
    sc = small_sequence(n_cams=12, seed=8)
    N, bi, bl, bs, diag, S = reduced_blocks(sc, 1e-12)
    Z = og.gauge_basis(sc.R, sc.T)
    rel = np.linalg.norm(S @ Z) / (np.linalg.norm(S) * np.linalg.norm(Z))
    assert rel < 1e-7
    assert np.linalg.matrix_rank(Z) == 7
