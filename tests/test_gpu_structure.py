"""The structure v3dba_create builds on the device (point-major order, camera lists, camera-pair
blocks and their observation pairs) equals the CPU restatement exactly, for ordered and shuffled
observations, cameras without observations and repeated (camera, point) observations."""
import numpy as np
import pytest

from oracle.structure import structure as cpu_structure
from v3dsfmtoolkit_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def check(sc):
    h = capi.Handle.from_scene(sc)
    g = h.structure()
    c = cpu_structure(sc.n_cams, sc.view, sc.point)
    for k in c:
        assert np.array_equal(g[k], c[k]), k
    h.close()


def test_point_major_scene():
    check(scenes.circle_scene(seed=4))


def test_shuffled_observations():
    sc = scenes.sequence_scene(n_cams=30, n_points=3000, mode=scenes.FULL_BUNDLE_METRIC, seed=6)
    order = np.random.default_rng(1).permutation(sc.n_obs)
    sc.view, sc.point, sc.meas = sc.view[order], sc.point[order], sc.meas[order]
    check(sc)


def test_camera_without_observations_and_repeats():
    sc = scenes.circle_scene(n_cams=9, n_points=400, seed=9)
    keep = sc.view != 4
    sc.view, sc.point, sc.meas = sc.view[keep], sc.point[keep], sc.meas[keep]
    # repeat a few observations (same camera, same point)
    rep = np.arange(0, sc.n_obs, 97)
    sc.view = np.concatenate([sc.view, sc.view[rep]])
    sc.point = np.concatenate([sc.point, sc.point[rep]])
    sc.meas = np.concatenate([sc.meas, sc.meas[rep] + 0.1])
    check(sc)


def test_large_scene_pair_counts():
    sc = scenes.cluster_scene(n_groups=3, cams_per_group=40, n_points=20000, seed=3)
    h = capi.Handle.from_scene(sc)
    g = h.structure()
    lens = np.bincount(sc.point, minlength=sc.n_points)
    # every point contributes, per observation k, the observations m with camera(m) >= camera(k)
    expect = 0
    order = np.argsort(sc.point, kind="stable")
    v = sc.view[order]
    start = 0
    for L in lens:
        cams = v[start:start + L]
        expect += int((cams[None, :] >= cams[:, None]).sum())
        start += L
    assert g["pr_k"].size == expect
    assert np.all(np.diff(g["b_ptr"]) >= 0) and g["b_ptr"][-1] == expect
    c = cpu_structure(sc.n_cams, sc.view, sc.point)
    for k in ("o_orig", "c_ptr", "c_obs", "b_i", "b_l", "b_ptr"):
        assert np.array_equal(g[k], c[k]), k
