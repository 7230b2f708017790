"""Rotation averaging on the GPU (v3dba_refine_consistent_rotations / v3dba_rotations_*) against
the reference's refineConsistentRotations: golden fixtures generated from the reference compiled
from its sources, and the bit-exact C restatement on larger seeded graphs.

Tolerances: the GPU sums the 3x3 normal blocks, gradients and costs in a different order (and
with fused multiply-adds), so costs agree to rounding (1e-9 relative at the first
linearisation, 1e-6 at the end) and rotations to 1e-5 (entries are at most 1 in magnitude).  The
late iterations of this slowly converging LM decide on cost differences near rounding, so the
relinearisation count may differ by a few; the exit status must be the same."""
import numpy as np
import pytest

from oracle.bindings import Restatement
from v3dsfmtoolkit_b200 import capi, scenes
from tests.helpers import load_rotation_golden, rotation_golden_names

pytestmark = pytest.mark.gpu


def _check_against(R, r, R_ref, trace_ref, status_ref, n_relin_ref):
    assert r.status == status_ref
    assert abs(r.initial_cost - trace_ref[0]) <= 1e-9 * max(trace_ref[0], 1e-300) + 1e-25
    assert abs(r.cost - trace_ref[-1]) <= 1e-6 * max(trace_ref[-1], 1e-300) + 1e-25
    assert np.abs(R - R_ref).max() < 1e-5
    assert abs(r.n_relinearizations - n_relin_ref) <= max(3, n_relin_ref // 10)


@pytest.mark.parametrize("name", rotation_golden_names())
def test_refine_consistent_rotations_matches_reference_fixture(name):
    graph, g = load_rotation_golden(name)
    R, r = capi.refine_consistent_rotations(graph.rel, graph.pairs, graph.R0)
    _check_against(R, r, g["R"], g["trace"], int(g["status"]), len(g["trace"]))


@pytest.mark.parametrize("n_views,n_pairs,outliers", [(2000, 40000, 0.0), (1000, 30000, 0.05)])
def test_large_graph_matches_restatement(n_views, n_pairs, outliers):
    graph = scenes.rotation_graph(n_views=n_views, n_pairs=n_pairs, seed=n_views, outlier_frac=outliers)
    Ro, info = Restatement().rotations_minimize(graph)
    R, r = capi.refine_consistent_rotations(graph.rel, graph.pairs, graph.R0)
    _check_against(R, r, Ro, info["trace_cost"], info["status"], info["n_relinearizations"])
    assert np.abs(R @ np.transpose(R, (0, 2, 1)) - np.eye(3)).max() < 1e-12


def test_handle_is_deterministic_and_resettable():
    graph = scenes.rotation_graph(n_views=500, n_pairs=8000, seed=7)
    h = capi.Rotations.from_graph(graph)
    c0 = h.cost()
    r1 = h.minimize()
    R1 = h.get()
    assert h.cost() == pytest.approx(r1.cost, rel=1e-12)
    h.reset()
    assert h.cost() == c0
    r2 = h.minimize()
    assert np.array_equal(h.get(), R1)
    assert (r1.status, r1.iterations, r1.n_relinearizations, r1.cost) == (r2.status, r2.iterations,
                                                                           r2.n_relinearizations, r2.cost)
    assert r1.device_ms > 0.0
    h.set(graph.R0)
    assert h.cost() == c0
    h.close()


def test_cost_matches_restatement():
    graph = scenes.rotation_graph(n_views=300, n_pairs=5000, seed=9, outlier_frac=0.1)
    h = capi.Rotations.from_graph(graph)
    assert h.cost() == pytest.approx(Restatement().rotations_cost(graph, graph.R0), rel=1e-12)


def test_options_and_stop_cost():
    graph, g = load_rotation_golden("rot_graph")
    _, r0 = capi.refine_consistent_rotations(graph.rel, graph.pairs, graph.R0, max_iterations=0)
    assert r0.status == capi.STATUS_TIMEOUT and r0.iterations == 0 and r0.n_relinearizations == 0
    _, r5 = capi.refine_consistent_rotations(graph.rel, graph.pairs, graph.R0, max_iterations=5)
    assert r5.iterations == 5 and r5.status == capi.STATUS_TIMEOUT
    target = float(g["trace"][10])
    _, rs = capi.refine_consistent_rotations(graph.rel, graph.pairs, graph.R0, stop_cost=target)
    assert rs.reached_stop_cost == 1 and rs.cost <= target and rs.iterations < int(g["iterations"])


def test_invalid_inputs_are_rejected():
    graph = scenes.rotation_graph(n_views=10, n_pairs=20, seed=1)
    bad = graph.pairs.copy()
    bad[3, 1] = 10
    with pytest.raises(capi.V3dbaError):
        capi.refine_consistent_rotations(graph.rel, bad, graph.R0)
    rel = graph.rel.copy()
    rel[2, 1, 1] = np.nan
    with pytest.raises(capi.V3dbaError):
        capi.refine_consistent_rotations(rel, graph.pairs, graph.R0)


def test_empty_problems():
    R, r = capi.refine_consistent_rotations(np.zeros((0, 3, 3)), np.zeros((0, 2), np.int32), np.zeros((0, 3, 3)))
    assert R.shape == (0, 3, 3) and r.status == capi.STATUS_CONVERGED
    R0 = scenes.rotation_graph(n_views=5, n_pairs=4, seed=2).R0
    R, r = capi.refine_consistent_rotations(np.zeros((0, 3, 3)), np.zeros((0, 2), np.int32), R0)
    assert r.status == capi.STATUS_CONVERGED and np.array_equal(R, R0)


def test_group_sizes_agree_and_autotune_picks_one():
    graph = scenes.rotation_graph(n_views=800, n_pairs=12000, seed=12)
    h = capi.Rotations.from_graph(graph)
    out = []
    for G in (4, 8, 16, 32):
        h.set_group(G)
        h.reset()
        r = h.minimize()
        out.append((r, h.get()))
    r0, R0 = out[0]
    for r, R in out[1:]:
        assert r.status == r0.status
        assert abs(r.cost - r0.cost) <= 1e-9 * r0.cost
        assert np.abs(R - R0).max() < 1e-8
    h.reset()
    c = h.cost()
    assert h.autotune() in (4, 8, 16, 32)
    assert h.cost() == pytest.approx(c, rel=1e-12)
    with pytest.raises(capi.V3dbaError):
        h.set_group(3)

