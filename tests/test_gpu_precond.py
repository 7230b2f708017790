"""Learned PCG preconditioner and gauge coarse space on the GPU: features, network outputs, loss
and weight gradients against the CPU oracle; BF16 inference against the FP32 path; training;
PCG iteration cuts; and the LM loop with the learned preconditioner against block-Jacobi as
fallback and check."""
import os

import numpy as np
import pytest

from oracle import precond_gnn as og
from precond_cases import converged_system, dense_pcg, reduced_blocks, small_sequence
from v3dsfmtoolkit_b200 import capi, precond, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    N, bi, bl, bs, diag, S = reduced_blocks(small_sequence(n_cams=12, seed=5), 1e-6)
    pset = capi.PrecondSet()
    pset.add_blocks(N, bi, bl, bs)
    g = og.Graph(N, bi, bl)
    xe, xn, cinv = og.features(g, bs, diag)
    return pset, g, xe, xn, cinv


def weights_with_output(seed, scale=0.05):
    rng = np.random.default_rng(seed)
    m = capi.PrecondModel(seed=seed)
    w = m.weights().astype(np.float64)
    o, k, n = og.LAYOUT["out"]
    w[o:o + (k + 1) * n] = rng.uniform(-scale, scale, size=(k + 1) * n)
    return w


def test_features_match_oracle(case):
    pset, g, xe, xn, cinv = case
    ea, eb, xe_g, xn_g, cinv_g = pset.features(0)
    assert np.array_equal(ea, g.ea) and np.array_equal(eb, g.eb)
    assert np.max(np.abs(xe_g - xe)) < 1e-4 * max(1.0, np.max(np.abs(xe)))
    assert np.allclose(xn_g, xn, rtol=1e-4, atol=1e-5)
    assert np.allclose(cinv_g, cinv, rtol=1e-4, atol=1e-6 * np.max(np.abs(cinv)))


def test_loss_and_weight_gradient_match_oracle(case):
    """FP32 forward/backward kernels against the FP64 oracle on the GPU's own features."""
    pset, g, _, _, _ = case
    _, _, xe_g, xn_g, _ = pset.features(0)
    xe, xn = xe_g.astype(np.float64), xn_g.astype(np.float64)
    m = capi.PrecondModel(weights_with_output(7).astype(np.float32))
    w32 = m.weights().astype(np.float64)
    loss_g, grad_g = m.loss_grad(pset, 0, probe_seed=99)
    loss_o, grad_o, coef_o = og.loss_and_grad(w32, g, xe, xn, 99)
    assert loss_g == pytest.approx(loss_o, rel=2e-4)
    coef_g = m.coefficients(pset, 0, bf16=False)
    assert np.max(np.abs(coef_g - coef_o)) < 1e-4 * max(1.0, np.max(np.abs(coef_o)))
    for name, (o, k, n) in og.LAYOUT.items():
        a, b = grad_g[o:o + (k + 1) * n], grad_o[o:o + (k + 1) * n]
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert err < 2e-3, (name, err)


def test_bf16_inference_follows_fp32(case):
    pset, _, _, _, _ = case
    m = capi.PrecondModel(weights_with_output(3, scale=0.2).astype(np.float32))
    c32 = m.coefficients(pset, 0, bf16=False)
    c16 = m.coefficients(pset, 0, bf16=True)
    assert np.max(np.abs(c16 - c32)) < 0.03 * max(1.0, np.max(np.abs(c32)))


def test_training_lowers_the_loss_and_is_deterministic():
    pset = capi.PrecondSet()
    for s, lam in [(11, 1e-5), (12, 1e-7), (13, 1e-8)]:
        N, bi, bl, bs, _, _ = reduced_blocks(small_sequence(n_cams=14, seed=s), lam)
        pset.add_blocks(N, bi, bl, bs)
    m1, h1 = precond.train(pset, epochs=25, lr=1e-3, seed=4)
    m2, h2 = precond.train(pset, epochs=25, lr=1e-3, seed=4)
    assert h1[-1] < h1[0]
    assert np.array_equal(h1, h2) and np.array_equal(m1.weights(), m2.weights())


def test_untrained_factor_cuts_pcg_iterations():
    """c = 1 (first-order FSAI factor) needs far fewer iterations than block-Jacobi; the GPU's
    block-Jacobi count matches the oracle's dense PCG within a few iterations."""
    from oracle.bindings import Restatement
    sc = scenes.sequence_scene(n_cams=60, n_points=6000, mode=scenes.FULL_BUNDLE_METRIC, seed=8, outlier_frac=0.0)
    N, bi, bl, bs, diag, S = reduced_blocks(sc, 1e-8)
    pset = capi.PrecondSet()
    pset.add_blocks(N, bi, bl, bs)
    it = pset.pcg_iterations(0, capi.PrecondModel(seed=0), tol=1e-6, max_iter=3000, rhs_seed=5)
    assert it["jacobi_gauge"] is None and it["learned_gauge"] is None   # no camera frames
    assert it["learned"] * 1.6 < it["jacobi"], it
    rng = np.random.default_rng(0)
    _, it_o = Restatement().pcg(S, rng.normal(size=6 * N), 6, rel_tol=1e-6, max_iter=3000)
    assert abs(it["jacobi"] - it_o) <= max(3, 0.1 * it_o)


def test_gauge_space_cuts_pcg_iterations_at_small_damping():
    """At the damping of a converged LM run the 7 gauge motions are the smallest eigenvectors:
    the gauge coarse space removes them (block-Jacobi + gauge beats block-Jacobi)."""
    sc = scenes.sequence_scene(n_cams=60, n_points=6000, mode=scenes.FULL_BUNDLE_METRIC, seed=4, outlier_frac=0.0)
    h = capi.Handle.from_scene(sc)
    r = h.minimize(max_iterations=20, solver=capi.SOLVER_PCG)
    pset = capi.PrecondSet()
    pset.capture(h, r.lambda_)
    it = pset.pcg_iterations(0, capi.PrecondModel(seed=0), tol=1e-6, max_iter=3000, rhs_seed=2)
    assert it["jacobi_gauge"] < it["jacobi"], it
    assert it["learned_gauge"] < it["learned"], it


@pytest.mark.parametrize("lam_rel", [1e-10, 1e-12])
def test_gauge_space_matches_dense_oracle_pcg(lam_rel):
    """PCG iteration counts of block-Jacobi and block-Jacobi + gauge space on a converged-state
    system follow the oracle's dense FP64 PCG with the same preconditioners (different seeded
    right-hand sides, so within 15%)."""
    N, bi, bl, bs, diag, S, R, T = converged_system(lam_rel=lam_rel)
    pset = capi.PrecondSet()
    pset.add_blocks(N, bi, bl, bs, R, T)
    it = pset.pcg_iterations(0, None, tol=1e-6, max_iter=5000, rhs_seed=3)
    n = 6 * N
    Pinv = np.zeros((n, n))
    for i in range(N):
        Pinv[6 * i:6 * i + 6, 6 * i:6 * i + 6] = np.linalg.inv(S[6 * i:6 * i + 6, 6 * i:6 * i + 6])
    Z = og.gauge_basis(R.reshape(-1, 3, 3), T)
    Ec = np.linalg.inv(Z.T @ S @ Z)
    b = np.random.default_rng(0).normal(size=n)
    j_o = dense_pcg(S, b, lambda r: Pinv @ r)
    g_o = dense_pcg(S, b, lambda r: Pinv @ r + Z @ (Ec @ (Z.T @ r)))
    assert abs(it["jacobi"] - j_o) <= 0.15 * j_o, (it, j_o, g_o)
    assert abs(it["jacobi_gauge"] - g_o) <= 0.15 * g_o, (it, j_o, g_o)


def shipped_model():
    if not os.path.exists(precond.WEIGHTS):
        pytest.skip("no trained weights shipped")
    return capi.PrecondModel.load(precond.WEIGHTS)


def test_trained_model_cuts_pcg_iterations_on_held_out_systems():
    """Held-out seeds (never used for training), systems captured from the adjuster's own LM
    runs, solved with the LM's own right-hand side: the learned factor at least halves the
    block-Jacobi PCG iterations and needs fewer than the untrained factor; with random
    right-hand sides (which excite the gauge motions) the gauge space adds to it."""
    m = shipped_model()
    m0 = capi.PrecondModel(seed=0)
    pset = capi.PrecondSet()
    for s in (990001, 990002, 990003, 990004):
        precond.capture(pset, precond.training_scenes(s, n_min=100, n_max=400), 3)
    t = precond.summarize(precond.evaluate(pset, m))
    u = precond.summarize(precond.evaluate(pset, m0))
    assert t["learned_iterations"] * 2 <= t["jacobi_iterations"], t
    assert t["learned_iterations"] < u["learned_iterations"], (t, u)
    r = precond.summarize(precond.evaluate(pset, m, rhs_seed=1))
    assert r["learned_gauge_iterations"] < r["learned_iterations"], r


def test_lm_with_learned_preconditioner_matches_block_jacobi():
    """FP64 blocks: the LM loop with the learned preconditioner reaches the cost of the
    block-Jacobi run within 1e-6 relative with at most half its PCG iterations; block-Jacobi
    is the check."""
    m = shipped_model()
    sc = scenes.cluster_scene(n_groups=4, cams_per_group=50, n_points=30000, seed=990011)
    hj = capi.Handle.from_scene(sc)
    rj = hj.minimize(max_iterations=40, solver=capi.SOLVER_PCG, precision=capi.PRECISION_FP64)
    cj = hj.cost()
    hl = capi.Handle.from_scene(sc)
    hl.set_precond_model(m)
    rl = hl.minimize(max_iterations=60, solver=capi.SOLVER_PCG, precision=capi.PRECISION_FP64,
                     preconditioner=capi.PRECOND_LEARNED, stop_cost=cj * (1 + 1e-6))
    assert hl.cost() <= cj * (1 + 1e-6)
    assert rl.pcg_iterations * 2 <= rj.pcg_iterations, (rl.pcg_iterations, rj.pcg_iterations)


def test_lm_mixed_precision_with_learned_preconditioner_reaches_the_same_cost():
    """Mixed precision: FP32 blocks can break the learned solve down (block-Jacobi then
    re-solves the trial); the run still reaches the block-Jacobi run's cost."""
    m = shipped_model()
    sc = scenes.cluster_scene(n_groups=4, cams_per_group=50, n_points=30000, seed=990011)
    hj = capi.Handle.from_scene(sc)
    hj.minimize(max_iterations=40, solver=capi.SOLVER_PCG)
    cj = hj.cost()
    hl = capi.Handle.from_scene(sc)
    hl.set_precond_model(m)
    rl = hl.minimize(max_iterations=60, solver=capi.SOLVER_PCG, preconditioner=capi.PRECOND_LEARNED,
                     stop_cost=cj * (1 + 1e-6))
    assert hl.cost() <= cj * (1 + 1e-6)
    assert rl.pcg_iterations > 0


def test_learned_without_model_is_rejected():
    sc = scenes.circle_scene(n_cams=8, n_points=300, seed=1)
    h = capi.Handle.from_scene(sc)
    with pytest.raises(capi.V3dbaError):
        h.minimize(max_iterations=3, solver=capi.SOLVER_PCG, preconditioner=capi.PRECOND_LEARNED)
