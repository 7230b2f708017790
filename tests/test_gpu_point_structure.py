"""BundlePointStructure on the GPU (v3dba_bundle_point_structure, v3dba_create_point_structure)
against the reference's own BundlePointStructure (V3D/include/Geometry/v3d_mviewutilities.h:
132-205, compiled in oracle/_ref): the flat bundle-adjustment inputs of a reconstruction and the
write-back into it, both createFromScratch branches, bit for bit."""
import numpy as np
import pytest

from oracle.bindings import Reference, reference_available
from v3dsfmtoolkit_b200 import capi

pytestmark = pytest.mark.gpu


def random_tracks(n, max_len, seed, n_views=40):
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, max_len + 1, size=n)
    ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    K = int(ptr[-1])
    return dict(track_ptr=ptr, pos=rng.normal(scale=10.0, size=(n, 3)), view=rng.integers(0, n_views, K).astype(np.int32),
                id=rng.integers(-1, 100000, K).astype(np.int32),
                mpos=(rng.uniform(0, 640, size=(K, 2))).astype(np.float32))


CASES = {
    "mixed": random_tracks(3000, 8, 1),
    "long": random_tracks(200, 300, 2),
    "all_short": random_tracks(500, 1, 3),
    "empty": dict(track_ptr=np.zeros(1, np.int32), pos=np.zeros((0, 3)), view=np.zeros(0, np.int32),
                  id=np.zeros(0, np.int32), mpos=np.zeros((0, 2), np.float32)),
    "no_measurements": dict(track_ptr=np.zeros(6, np.int32), pos=np.ones((5, 3)), view=np.zeros(0, np.int32),
                            id=np.zeros(0, np.int32), mpos=np.zeros((0, 2), np.float32)),
}


@pytest.fixture(scope="module")
def ref():
    if not reference_available():
        pytest.skip("compiled reference not present")
    return Reference()


def _same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        assert a[k].dtype == b[k].dtype or a[k].size == 0, k
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("n_required", [-1, 0, 1, 2, 5])
def test_bundle_point_structure_matches_reference(ref, case, n_required):
    tracks = CASES[case]
    _same(capi.bundle_point_structure(tracks, n_required), ref.bundle_point_structure(tracks, n_required))


@pytest.mark.parametrize("case", list(CASES))
def test_create_point_structure_from_scratch_matches_reference(ref, case):
    tracks = CASES[case]
    bps = ref.bundle_point_structure(tracks, 2)
    bps["points3d"] = bps["points3d"] * 1.5 + 0.25        # as an adjustment would move them
    bps["measurements"] = bps["measurements"] + 1e-3
    _same(capi.create_point_structure(bps, from_scratch=True), ref.create_point_structure(bps, True))


@pytest.mark.parametrize("case", list(CASES))
def test_create_point_structure_in_place_matches_reference(ref, case):
    tracks = CASES[case]
    bps = ref.bundle_point_structure(tracks, 3)
    bps["points3d"] = bps["points3d"] - 2.0
    bps["measurements"] = bps["measurements"] * 0.5 + 1.0 / 3.0   # not representable in float: rounding
    got = capi.create_point_structure(bps, from_scratch=False, tracks=tracks)
    want = ref.create_point_structure(bps, False, tracks)
    _same(got, want)
    # the tracks that were not kept are unchanged
    kept = np.zeros(len(tracks["pos"]), bool)
    kept[bps["xs_indices"]] = True
    np.testing.assert_array_equal(got["pos"][~kept], tracks["pos"][~kept])


def test_round_trip_through_a_minimize_input():
    """The flat arrays feed v3dba_create directly (points3d, measurements, corresponding_view /
    corresponding_point are the optimizer's inputs) and write back from scratch unchanged."""
    tracks = random_tracks(1000, 6, 9)
    bps = capi.bundle_point_structure(tracks, 2)
    back = capi.create_point_structure(bps, from_scratch=True)
    again = capi.bundle_point_structure(back, 2)
    for k in ("points3d", "measurements", "measurement_ids", "corresponding_view", "corresponding_point"):
        np.testing.assert_array_equal(again[k], bps[k])
    np.testing.assert_array_equal(again["xs_indices"], np.arange(len(bps["points3d"])))


def test_invalid_inputs_are_rejected():
    bad = dict(CASES["mixed"])
    bad["track_ptr"] = bad["track_ptr"].copy()
    bad["track_ptr"][5] = bad["track_ptr"][4] - 1
    with pytest.raises(capi.V3dbaError) as e:
        capi.bundle_point_structure(bad, 2)
    assert e.value.code == capi.ERR_INVALID_INPUT
    bps = capi.bundle_point_structure(CASES["mixed"], 2)
    bps["corresponding_point"] = bps["corresponding_point"].copy()
    bps["corresponding_point"][0] = len(bps["points3d"])
    with pytest.raises(capi.V3dbaError) as e:
        capi.create_point_structure(bps, from_scratch=True)
    assert e.value.code == capi.ERR_INVALID_INPUT


def test_empty_write_back_accepts_null_arrays():
    """A structure that kept no track (n_required above every track length, or negative) writes
    back an empty reconstruction from scratch; the arrays with nothing to hold may be NULL, as
    data() of an empty std::vector is."""
    import ctypes as C
    lib = capi.library()
    ptr = np.full(1, -7, np.int32)
    rc = lib.v3dba_create_point_structure(1, 0, 0, None, None, None, None, None, None, 0,
                                          ptr.ctypes.data_as(C.POINTER(C.c_int)), None, None, None, None)
    assert rc == capi.OK
    assert ptr[0] == 0
    # in place over zero tracks: nothing is read or written but track_ptr[0]
    rc = lib.v3dba_create_point_structure(0, 0, 0, None, None, None, None, None, None, 0,
                                          ptr.ctypes.data_as(C.POINTER(C.c_int)), None, None, None, None)
    assert rc == capi.OK
