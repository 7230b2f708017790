"""Device allocation failures end the call with a clean error code (failure case iv of the
reference's error convention: no exception, an int code from the C-ABI) and leave the library
usable.  The failure is injected on the host (v3dba_debug_fail_allocation) in front of the
allocation call, so no GPU ever faults."""
import numpy as np
import pytest

from v3dsfmtoolkit_b200 import capi, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _injection_off():
    capi.debug_fail_allocation(-1)
    yield
    capi.debug_fail_allocation(-1)


def _clean_run(sc, iters):
    h = capi.Handle.from_scene(sc)
    r = h.minimize(max_iterations=iters, precision=capi.PRECISION_FP64)
    p = h.get_params()
    h.close()
    return r, p


@pytest.mark.parametrize("solver", [capi.SOLVER_CHOLESKY, capi.SOLVER_PCG])
def test_every_allocation_of_create_and_minimize_fails_cleanly(solver):
    sc = scenes.circle_scene(n_cams=6, n_points=150, seed=7)
    r_ref, p_ref = _clean_run(sc, 10)
    failed_create = failed_minimize = 0
    for k in range(400):
        capi.debug_fail_allocation(k)
        try:
            h = capi.Handle.from_scene(sc)
        except capi.V3dbaError as e:
            assert e.code == capi.ERR_OUT_OF_MEMORY, e
            failed_create += 1
            continue
        try:
            r = h.minimize(max_iterations=10, precision=capi.PRECISION_FP64, solver=solver)
        except capi.V3dbaError as e:
            assert e.code == capi.ERR_OUT_OF_MEMORY, e
            failed_minimize += 1
            # the handle stays valid: with the injection spent, the same call now succeeds
            r = h.minimize(max_iterations=10, precision=capi.PRECISION_FP64, solver=solver)
        else:
            capi.debug_fail_allocation(-1)
            h.close()
            break
        h.close()
    else:
        pytest.fail("the injected failure never ran out")
    assert failed_create > 5 and failed_minimize >= 1
    # nothing left behind: a fresh run gives the same result as before the injections
    r2, p2 = _clean_run(sc, 10)
    assert (r2.status, r2.iterations) == (r_ref.status, r_ref.iterations)
    for a, b in zip(p2, p_ref):
        np.testing.assert_array_equal(a, b)


def test_batch_create_fails_cleanly():
    trips = scenes.triplet_batch(n_triplets=8, min_points=20, max_points=40, seed=3)
    for k in range(3):
        capi.debug_fail_allocation(k)
        with pytest.raises(capi.V3dbaError) as e:
            capi.Batch(trips)
        assert e.value.code == capi.ERR_OUT_OF_MEMORY
    capi.debug_fail_allocation(-1)
    b = capi.Batch(trips)
    res, _ = b.minimize(max_iterations=5)
    assert all(r.iterations > 0 for r in res)
    b.close()
