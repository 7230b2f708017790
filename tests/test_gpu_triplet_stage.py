"""The triplet stage on the GPU (v3dba_triplet_stage: triangulation and filtering of every track,
survival tests, batched adjustment) against the reference's triplet stage (golden fixture) and
the restatement on a larger seeded batch.

Tolerances: the filter reproduces the reference's float arithmetic, so the verdicts, surviving
counts and kept-measurement flags must be identical; the linear triangulation uses the device's
hypot (to 1 ulp of the C library's), the adjustment is FP64 with a different summation order:
points and cameras within 1e-7, the adjustment's status and iteration count the same."""
import numpy as np
import pytest

from oracle import triplet_stage as ots
from v3dsfmtoolkit_b200 import capi, scenes
from tests.helpers import load_triplet_stage_golden

pytestmark = pytest.mark.gpu


def _compare(a, b, tol=1e-7):
    assert a["verdict"] == b["verdict"] and a["n_points"] == b["n_points"]
    assert np.array_equal(a["kept"], b["kept"])
    if b["verdict"] == capi.TRIPLET_ACCEPTED:
        assert a["status"] == b["status"] and a["iterations"] == b["iterations"]
        assert abs(a["cost"] - b["cost"]) <= 1e-6 * max(abs(b["cost"]), 1e-300)
    assert np.abs(a["R"] - b["R"]).max() < tol and np.abs(a["T"] - b["T"]).max() < tol
    xa, xb = np.asarray(a["X"]), np.asarray(b["X"])
    assert np.array_equal(np.isnan(xa), np.isnan(xb))
    fin = ~np.isnan(xb)
    if fin.any():
        assert np.abs(xa[fin] - xb[fin]).max() <= tol * max(1.0, np.abs(xb[fin]).max())


def test_triplet_stage_matches_reference_fixture():
    trips, outs = load_triplet_stage_golden()
    res = capi.triplet_stage(trips)
    for a, b in zip(res, outs):
        _compare(a, b)


def test_triplet_stage_batch_matches_restatement():
    trips = scenes.triplet_stage_batch(n_triplets=64, seed=5, max_tracks=400)
    res = capi.triplet_stage(trips)
    for t, a in zip(trips, res):
        _compare(a, ots.stage(t))


def test_options_change_the_verdicts():
    trips = scenes.triplet_stage_batch(n_triplets=16, seed=6, max_tracks=300)
    strict = capi.triplet_stage(trips, min_points=10**6)
    assert all(r["verdict"] == capi.TRIPLET_TOO_FEW_POINTS for r in strict)
    loose = capi.triplet_stage(trips, max_reproj_error=1e9, min_points=0, min_point_ratio=0.0)
    for t, r in zip(trips, loose):
        lens = np.diff(t.track_ptr)
        assert r["verdict"] == capi.TRIPLET_ACCEPTED and r["n_points"] == int((lens >= 3).sum())
    for t, r in zip(trips, capi.triplet_stage(trips, max_iterations=0)):
        if r["verdict"] == capi.TRIPLET_ACCEPTED:
            assert r["iterations"] == 0 and np.array_equal(r["R"], t.R)


def test_invalid_triplets_are_rejected():
    t = scenes.triplet_stage_batch(n_triplets=1, seed=7, max_tracks=60)[0]
    bad = scenes.TripletTracks(t.R, t.T, t.focal, t.track_ptr, np.where(t.view == 2, 3, t.view).astype(np.int32), t.pos)
    with pytest.raises(capi.V3dbaError):
        capi.triplet_stage([bad])
    pos = t.pos.copy()
    pos[0, 0] = np.nan
    with pytest.raises(capi.V3dbaError):
        capi.triplet_stage([scenes.TripletTracks(t.R, t.T, t.focal, t.track_ptr, t.view, pos)])


def test_flat_entry_point_matches_the_per_triplet_one():
    trips = scenes.triplet_stage_batch(n_triplets=40, seed=8, max_tracks=300)
    per = capi.triplet_stage(trips)
    flat = capi.triplet_stage_flat(capi.concat_triplets(trips))
    g = m = 0
    for i, (t, r) in enumerate(zip(trips, per)):
        assert flat["verdict"][i] == r["verdict"] and flat["n_points"][i] == r["n_points"]
        assert np.array_equal(flat["X"][g:g + t.n_tracks], r["X"], equal_nan=True)
        nm = int(t.track_ptr[-1])
        assert np.array_equal(flat["kept"][m:m + nm], r["kept"])
        if r["verdict"] == capi.TRIPLET_ACCEPTED:
            assert flat["status"][i] == r["status"] and np.array_equal(flat["R"][i], r["R"])
        g += t.n_tracks
        m += nm

