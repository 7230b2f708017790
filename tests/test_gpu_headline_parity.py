"""Parity on the headline scene (200-camera distortion sequence, 50,000 points, ~375k
observations, CommonInternals RADIAL_TANGENTIAL, Huber 1 px) against the reference optimizer
compiled from its sources (oracle/_ref), at full size.

The reference's own 100-iteration run does not converge: at its last iterations the Huber
re-weighting still lowers the cost by ~5e-7 per relinearisation, along directions where the
parameters are nearly free (points close to the direction of travel, whose depth the short
baselines barely fix).  Its final parameters there are not a property of the problem but of the
path: the reference started with tau * (1 + 1e-12) instead of tau ends with the same cost to
2e-8 but points 2e-3 apart (relative to the scene's extent), and with tau * (1 + 2e-12) on
another path (31 rejected steps instead of 23), 2.3e-5 above in cost and 0.7 apart in points.
The reference's spread is estimated from its own runs with tau * (1 + k * 1e-12), k = 1 .. 7 (a
handful of samples of a chaotic path: fewer would understate it).  So the comparisons here are:
  * the first iterations, where the two implementations take the same accept / reject
    decisions: cost and parameters to tight tolerances;
  * the 100-iteration run and the runs that stop on the reference's final cost: same status,
    cost within the spread of the reference's own tau-perturbed runs, and gauge-aligned
    parameters no further from the nearest of the reference's end states than the reference's
    own perturbed runs are from its unperturbed one.
"""
import json
import multiprocessing as mp
import os

import numpy as np
import pytest

from v3dsfmtoolkit_b200 import capi, scenes
from tests.helpers import param_rel, similarity_align

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TAU_STEP = 1e-12
PREFIX_ITERATIONS = 40   # iterations over which both implementations take the same LM decisions


def _reference_run(args):
    """One reference minimize() in a spawned process (no CUDA there): (params, cost, info)."""
    k, iters = args
    from oracle.bindings import Reference
    sc = scenes.sequence_scene()
    ref = Reference()
    params, info = ref.minimize(sc, max_iterations=iters, tau=1e-3 * (1 + k * TAU_STEP))
    return params, ref.cost(sc, params), {"status": info["status"], "iterations": info["iterations"],
                                           "n_rejected": info["n_rejected"]}


N_PERTURBED = 8   # the reference's own runs with tau * (1 + k * 1e-12), k = 0 .. N_PERTURBED - 1


@pytest.fixture(scope="module")
def reference_runs():
    from oracle.bindings import reference_available
    if not reference_available():
        pytest.skip("compiled reference not present")
    jobs = [(k, 100) for k in range(N_PERTURBED)] + [(0, PREFIX_ITERATIONS)]
    with mp.get_context("spawn").Pool(min(len(jobs), max(os.cpu_count() or 1, 1))) as pool:
        out = pool.map(_reference_run, jobs)
    return {"perturbed": out[:N_PERTURBED], "prefix": out[N_PERTURBED]}


@pytest.fixture(scope="module")
def scene():
    sc = scenes.sequence_scene()
    ref = json.load(open(os.path.join(GOLDEN, "bench_reference.json")))["sequence200"]
    return sc, ref


def _nearest_reference(p, runs):
    """Gauge-aligned distance from p to the nearest of the reference's own end states (its runs
    under a 1e-12 change of tau end in several places of the nearly flat valley)."""
    return min(_aligned_error(p, q) for q, _, _ in runs)


def _aligned_error(p, q):
    """Max relative difference of (K, dist, R, T, X) after moving p's reconstruction onto q's by
    the best similarity (the gauge freedom of metric BA)."""
    K, R, T, d, X = p
    Kq, Rq, Tq, dq, Xq = q
    Ra, Ta, Xa = similarity_align(R, T, X, Rq, Tq, Xq)
    return param_rel((K, d, Ra, Ta, Xa), (Kq, dq, Rq, Tq, Xq))


def test_reference_runs_are_the_recorded_ones(reference_runs, scene):
    """The reference is deterministic: its unperturbed run here is the one the bench target was
    recorded from."""
    _, ref = scene
    _, c0, i0 = reference_runs["perturbed"][0]
    assert c0 == ref["cost"]
    assert (i0["status"], i0["iterations"], i0["n_rejected"]) == (ref["status"], 100, ref["n_rejected"])


def test_first_iterations_match_reference_tightly(reference_runs, scene):
    """Over the first iterations both take the same steps: FP64 cost to 1e-9 and parameters
    (raw, no gauge alignment) to 1e-6, same status and rejections."""
    sc, _ = scene
    p_ref, c_ref, i_ref = reference_runs["prefix"]
    h = capi.Handle.from_scene(sc)
    r = h.minimize(max_iterations=PREFIX_ITERATIONS, precision=capi.PRECISION_FP64)
    assert (r.status, r.iterations, r.n_rejected) == (i_ref["status"], i_ref["iterations"], i_ref["n_rejected"])
    assert abs(h.cost() - c_ref) <= 1e-9 * c_ref
    K, R, T, d, X = h.get_params()
    assert param_rel((K, d, R, T, X), (p_ref[0], p_ref[3], p_ref[1], p_ref[2], p_ref[4])) < 1e-6
    h.close()


def test_100_iterations_within_the_reference_spread(reference_runs, scene):
    """FP64 and mixed precision, 100 iterations: the reference's status (TIMEOUT), the cost no
    higher than the highest of the reference's tau-perturbed runs (1e-6) and not far below the
    lowest (a lower cost is a better minimum, so 1e-5 there), the gauge-aligned parameters no
    further from the nearest of the reference's runs than its perturbed runs are from its
    unperturbed one."""
    sc, _ = scene
    runs = reference_runs["perturbed"]
    p0, c0, i0 = runs[0]
    costs = [c for _, c, _ in runs]
    spread = max(_aligned_error(p, p0) for p, _, _ in runs[1:])
    assert spread > 1e-3   # the reference's final parameters move this much under a 1e-12 change of tau
    h = capi.Handle.from_scene(sc)
    for precision in (capi.PRECISION_FP64, capi.PRECISION_MIXED):
        h.reset_params()
        r = h.minimize(max_iterations=100, precision=precision)
        c = h.cost()
        err = _nearest_reference(h.get_params(), runs)
        print(f"precision {precision}: cost {(c - c0) / c0:+.3e} rel, rejections {r.n_rejected} "
              f"(reference {i0['n_rejected']}), aligned parameters {err:.3e} (reference spread {spread:.3e})")
        assert r.status == i0["status"] == capi.STATUS_TIMEOUT
        assert min(costs) * (1 - 1e-5) <= c <= max(costs) * (1 + 1e-6)
        assert err <= spread
    h.close()


def test_runs_to_the_reference_cost(reference_runs, scene):
    """The bench's step: minimize() until the reference's final cost (1e-6 relative), tau scaled by
    1 + k * 1e-12.  At least 6 of 8 runs in each precision reach it; their parameters are no
    further (gauge-aligned) from the nearest of the reference's runs than its perturbed runs are
    from its unperturbed one.  A run that stops
    with SMALL_UPDATE instead has entered a region where the reference's LM stalls as well: the
    reference started from that run's parameters also ends with SMALL_UPDATE without reaching
    the cost."""
    from oracle.bindings import Reference
    sc, _ = scene
    runs = reference_runs["perturbed"]
    p0, c0, _ = runs[0]
    spread = max(_aligned_error(p, p0) for p, _, _ in runs[1:])
    target = c0 * (1 + 1e-6)
    h = capi.Handle.from_scene(sc)
    for precision in (capi.PRECISION_FP64, capi.PRECISION_MIXED):
        reached = 0
        for k in range(8):
            h.reset_params()
            r = h.minimize(max_iterations=1000, precision=precision, stop_cost=target, tau=1e-3 * (1 + k * TAU_STEP))
            params = h.get_params()
            if r.reached_stop_cost:
                reached += 1
                err = _nearest_reference(params, runs)
                print(f"precision {precision} k {k}: reached in {r.iterations} iterations, aligned parameters "
                      f"{err:.3e} from the nearest reference run, {_aligned_error(params, p0):.3e} from the "
                      f"unperturbed one (reference spread {spread:.3e})")
                assert h.cost() <= target
                assert err <= spread
            else:
                assert r.status == capi.STATUS_SMALL_UPDATE
                assert h.cost() <= c0 * (1 + 1e-3)
                stalled = sc.copy()
                stalled.set_params(*params)
                rp, info = Reference().minimize(stalled, max_iterations=100)
                assert info["status"] == capi.STATUS_SMALL_UPDATE
                assert Reference().cost(stalled, rp) > target
        assert reached >= 6, (precision, reached)
    h.close()
