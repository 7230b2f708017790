"""Triplet stage oracle (test infrastructure): the numpy restatement (oracle/triplet_stage.py)
against the reference's triplet stage (tests/golden/triplets/stage.npz, generated from the
reference compiled from its sources) and, where that compiled reference is present, on fresh
triplets.  Triangulation and filtering are bit-exact; the adjustment runs on the C restatement
of the LM, equal to the reference's to rounding."""
import numpy as np
import pytest

from oracle import triplet_stage as ots
from oracle.bindings import Reference, reference_available
from v3dsfmtoolkit_b200 import scenes
from tests.helpers import load_triplet_stage_golden


@pytest.fixture(scope="module")
def golden():
    return load_triplet_stage_golden()


def test_fixture_covers_every_verdict(golden):
    _, outs = golden
    assert {o["verdict"] for o in outs} == {0, 1, 2}
    assert any(len(o["kept"]) == 0 for o in outs)


def _compare(a, b, x_tol=1e-9):
    assert a["verdict"] == b["verdict"] and a["n_points"] == b["n_points"]
    assert np.array_equal(a["kept"], b["kept"])
    assert a["status"] == b["status"] and a["iterations"] == b["iterations"]
    assert abs(a["cost"] - b["cost"]) <= 1e-9 * max(abs(b["cost"]), 1e-300)
    assert np.abs(a["R"] - b["R"]).max() < 1e-9 and np.abs(a["T"] - b["T"]).max() < 1e-9
    xa, xb = np.asarray(a["X"]), np.asarray(b["X"])
    assert np.array_equal(np.isnan(xa), np.isnan(xb))
    fin = ~np.isnan(xb)
    if fin.any():
        assert np.abs(xa[fin] - xb[fin]).max() <= x_tol * max(1.0, np.abs(xb[fin]).max())


def test_restatement_matches_golden(golden):
    trips, outs = golden
    for t, o in zip(trips, outs):
        _compare(ots.stage(t), o)


def test_triangulation_and_filter_are_bit_exact(golden):
    trips, outs = golden
    for t, o in zip(trips, outs):
        if o["verdict"] == 0:
            continue    # refined points: compared with a tolerance above
        r = ots.stage(t)
        assert np.array_equal(np.nan_to_num(r["X"], nan=7.0), np.nan_to_num(o["X"], nan=7.0))


@pytest.mark.skipif(not reference_available(), reason="compiled reference not present")
def test_restatement_matches_reference_fresh_triplets():
    ref = Reference()
    for t in scenes.triplet_stage_batch(n_triplets=6, seed=77, max_tracks=200):
        _compare(ots.stage(t), ref.triplet_stage(t))
