"""The CPU oracle (test infrastructure): the C restatement pinned against the reference optimizer's
own outputs (golden fixtures generated from the reference compiled from its sources) and, where
the compiled reference is present, against fresh runs of it."""
import numpy as np
import pytest

from oracle.bindings import Reference, Restatement, reference_available
from v3dsfmtoolkit_b200 import scenes
from tests.helpers import golden_names, load_golden, param_rel, rel


@pytest.fixture(scope="module")
def orc():
    return Restatement()


@pytest.mark.parametrize("name", golden_names())
def test_restatement_linearization_matches_golden(orc, name):
    sc, g = load_golden(name)
    e, w, A, B, C = orc.linearize(sc)
    n = g["e"].shape[0]
    assert np.abs(e[:n] - g["e"]).max() <= 1e-12 * max(1.0, np.abs(g["e"]).max())
    np.testing.assert_allclose(w[:n], g["w"], rtol=1e-14, atol=0)
    assert rel(A[:n], g["A"]) < 1e-13
    assert rel(B[:n], g["B"]) < 1e-13
    if sc.dims[1]:
        assert rel(C[:n], g["C"]) < 1e-13


@pytest.mark.parametrize("name", golden_names())
def test_restatement_minimize_matches_golden(orc, name):
    sc, g = load_golden(name)
    params, info = orc.minimize(sc, max_iterations=int(g["max_iterations"]), nonvarying=tuple(g["nonvarying"]))
    assert info["status"] == int(g["status"])
    assert info["iterations"] == int(g["iterations"])
    assert info["n_rejected"] == int(g["n_rejected"])
    cost = orc.cost(sc, params)
    assert abs(cost - float(g["cost"])) <= 1e-8 * float(g["cost"])
    nt = min(len(info["trace_cost"]), len(g["trace_cost"]))
    assert rel(info["trace_cost"][:nt], g["trace_cost"][:nt]) < 1e-8
    assert param_rel((params[0], params[1], params[2], params[4]), (g["K"], g["R"], g["T"], g["X"])) < 1e-5


@pytest.mark.skipif(not reference_available(), reason="compiled reference not present")
@pytest.mark.parametrize("seed", [21, 22])
def test_restatement_matches_reference_fresh_seeds(orc, seed):
    ref = Reference()
    sc = scenes.circle_scene(n_cams=7, n_points=200, seed=seed)
    (pr, ir), (po, io) = ref.minimize(sc, max_iterations=40), orc.minimize(sc, max_iterations=40)
    assert ir["status"] == io["status"] and ir["iterations"] == io["iterations"]
    assert param_rel(pr, po) < 1e-8
    e1, _, A1, B1, _ = ref.linearize(sc)
    e2, _, A2, B2, _ = orc.linearize(sc)
    assert np.array_equal(e1, e2) or rel(e1, e2) < 1e-14
    assert rel(A1, A2) < 1e-14 and rel(B1, B2) < 1e-14


def test_reduced_system_solution_equals_full_normal_equations(orc):
    """One damped step through the point-eliminated system equals the solve of the full damped
    normal equations (what the reference's sparse LDL^T factors)."""
    sc = scenes.circle_scene(n_cams=5, n_points=60, seed=3)
    dA, dC = sc.dims
    bl = orc.normal_blocks(sc)
    lam = 0.37
    S, rhs, Vinv, fail = orc.reduced_system(sc, bl, lam)
    assert not fail
    da, f2 = orc.cholesky_solve(S, rhs)
    assert not f2
    # full system J^T J + lam I from the raw Jacobians
    e, w, A, B, _ = orc.linearize(sc)
    N, M = sc.n_cams, sc.n_points
    n = N * dA + M * 3
    J = np.zeros((2 * sc.n_obs, n))
    for k in range(sc.n_obs):
        i, j = sc.view[k], sc.point[k]
        J[2 * k:2 * k + 2, i * dA:(i + 1) * dA] = w[k] * A[k]
        J[2 * k:2 * k + 2, N * dA + 3 * j:N * dA + 3 * j + 3] = w[k] * B[k]
    r = -(w[:, None] * e).reshape(-1)
    H = J.T @ J + lam * np.eye(n)
    full = np.linalg.solve(H, J.T @ r)
    assert rel(da, full[:N * dA]) < 1e-9


def test_oracle_cholesky_rejects_indefinite(orc):
    S = np.array([[1.0, 2.0], [2.0, 1.0]])
    _, fail = orc.cholesky_solve(S, np.ones(2))
    assert fail


def test_oracle_pcg_converges(orc):
    rng = np.random.default_rng(0)
    A = rng.normal(size=(60, 60))
    S = A @ A.T + 60 * np.eye(60)
    b = rng.normal(size=60)
    x, it = orc.pcg(S, b, 6, rel_tol=1e-10, max_iter=500)
    assert it < 500
    assert rel(S @ x, b) < 1e-8


def test_reference_bundle_point_structure_round_trip():
    """The compiled reference's BundlePointStructure and createPointStructure (from scratch)
    invert each other on tracks that all pass the measurement threshold."""
    from oracle.bindings import Reference, reference_available
    if not reference_available():
        pytest.skip("compiled reference not present")
    rng = np.random.default_rng(4)
    lens = rng.integers(2, 6, size=100)
    ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    K = int(ptr[-1])
    tracks = dict(track_ptr=ptr, pos=rng.normal(size=(100, 3)), view=rng.integers(0, 9, K).astype(np.int32),
                  id=rng.integers(0, 999, K).astype(np.int32), mpos=rng.normal(size=(K, 2)).astype(np.float32))
    ref = Reference()
    bps = ref.bundle_point_structure(tracks, 2)
    back = ref.create_point_structure(bps, True)
    for k in tracks:
        np.testing.assert_array_equal(back[k], tracks[k])
    assert ref.bundle_point_structure(tracks, -1)["points3d"].shape[0] == 0   # size_t comparison
