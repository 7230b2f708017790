"""k_chol_levels (the level-scheduled tile Cholesky under a nested-dissection tile order) on the
GPU, through the C-ABI: dense solves of SPD systems with sequence-like and irregular tile
patterns against numpy (1e-10 relative, as for the column-by-column kernel), the two kernels
against each other, pivot failure, and a full LM run of a sequence scene on either kernel."""
import numpy as np
import pytest

from v3dsfmtoolkit_b200 import capi, scenes
from tests.test_chol_schedule import band_arrow, groups, random_pattern

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def spd_with_tiles(pat, n, seed):
    """SPD matrix of size n whose 64x64 tile pattern is (a subset of) pat."""
    rng = np.random.default_rng(seed)
    S = np.zeros((n, n))
    nt = pat.shape[0]
    for r in range(nt):
        for c in range(r + 1):
            if pat[r, c]:
                S[r * 64:(r + 1) * 64, c * 64:(c + 1) * 64] = 0.05 * rng.normal(size=(min(64, n - r * 64),
                                                                                      min(64, n - c * 64)))
    S = np.tril(S, -1)
    S = S + S.T
    S += np.diag(np.abs(S).sum(1) + 1.0)
    return S, rng.normal(size=n)


CASES = [
    ("band_arrow19", band_arrow(19), 19 * 64 - 9),
    ("band_arrow33", band_arrow(33, band=3), 33 * 64 - 40),
    ("random20", random_pattern(20, 0.15, 3), 20 * 64 - 1),
    ("groups24", groups(24, 6, 5), 24 * 64),
    ("small5", band_arrow(5), 5 * 64 - 30),
    ("blockdiag16", np.eye(16, dtype=bool), 16 * 64 - 3),          # one level
    ("arrow16", np.eye(16, dtype=bool) | (np.arange(16)[:, None] == 15), 16 * 64 - 7),  # two
]


@pytest.mark.parametrize("name,pat,n", CASES, ids=[c[0] for c in CASES])
def test_levels_solve_matches_numpy_and_column_kernel(name, pat, n, monkeypatch):
    S, b = spd_with_tiles(pat, n, seed=n)
    xr = np.linalg.solve(S, b)
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "levels")
    x_lv, fail = capi.dense_cholesky_solve(S, b)
    assert not fail
    assert rel(x_lv, xr) < 1e-10
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "steps")
    x_st, fail = capi.dense_cholesky_solve(S, b)
    assert not fail
    assert rel(x_lv, x_st) < 1e-11


def test_levels_solve_is_deterministic(monkeypatch):
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "levels")
    S, b = spd_with_tiles(band_arrow(19), 19 * 64 - 9, seed=1)
    x1, _ = capi.dense_cholesky_solve(S, b)
    x2, _ = capi.dense_cholesky_solve(S, b)
    assert np.array_equal(x1, x2)


def test_levels_report_indefinite(monkeypatch):
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "levels")
    S, b = spd_with_tiles(band_arrow(12), 12 * 64, seed=2)
    S[300, 300] = -5.0
    _, fail = capi.dense_cholesky_solve(S, b)
    assert fail


def test_sequence_scene_runs_on_the_level_schedule(monkeypatch):
    sc = scenes.sequence_scene(n_cams=120, n_points=12000, seed=3)
    h = capi.Handle.from_scene(sc)
    kind, n_levels, nt = h.cholesky_schedule()
    assert kind == "levels" and n_levels < nt
    r_lv = h.minimize(max_iterations=15, precision=capi.PRECISION_FP64)
    p_lv = h.get_params()
    h.close()
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "steps")
    h2 = capi.Handle.from_scene(sc)
    assert h2.cholesky_schedule()[0] == "steps"
    r_st = h2.minimize(max_iterations=15, precision=capi.PRECISION_FP64)
    p_st = h2.get_params()
    h2.close()
    assert r_lv.status == r_st.status and r_lv.iterations == r_st.iterations
    assert abs(r_lv.cost - r_st.cost) <= 1e-9 * r_st.cost
    for a, b in zip(p_lv, p_st):
        if a is not None:
            assert np.abs(a - b).max() <= 1e-7 * max(np.abs(b).max(), 1.0)


def test_stereo_rig_scene_runs_on_the_level_schedule(monkeypatch):
    sc = scenes.stereo_rig_scene(n_poses=150, n_points=12000, seed=4, window=6, outlier_frac=0.01)
    h = capi.Handle.from_scene(sc)
    kind, n_levels, nt = h.cholesky_schedule()
    assert kind == "levels" and n_levels < nt
    r_lv = h.minimize(max_iterations=12, precision=capi.PRECISION_FP64)
    p_lv = h.get_params()
    h.close()
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "steps")
    h2 = capi.Handle.from_scene(sc)
    r_st = h2.minimize(max_iterations=12, precision=capi.PRECISION_FP64)
    p_st = h2.get_params()
    h2.close()
    assert r_lv.status == r_st.status and r_lv.iterations == r_st.iterations
    assert abs(r_lv.cost - r_st.cost) <= 1e-9 * r_st.cost
    for a, b in zip(p_lv, p_st):
        if a is not None:
            assert np.abs(a - b).max() <= 1e-7 * max(np.abs(b).max(), 1.0)


def test_varying_intrinsics_scene_runs_on_the_level_schedule(monkeypatch):
    """VaryingInternals: 13 unknowns per camera, so the camera blocks straddle tiles differently
    and the band is wider than the 6-unknown sequences'."""
    sc = scenes.varying_scene(n_cams=150, n_points=15000, seed=2)
    h = capi.Handle.from_scene(sc)
    kind, n_levels, nt = h.cholesky_schedule()
    assert kind == "levels" and n_levels < nt
    r_lv = h.minimize(max_iterations=10, precision=capi.PRECISION_FP64)
    p_lv = h.get_params()
    h.close()
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "steps")
    h2 = capi.Handle.from_scene(sc)
    r_st = h2.minimize(max_iterations=10, precision=capi.PRECISION_FP64)
    p_st = h2.get_params()
    h2.close()
    assert r_lv.status == r_st.status and r_lv.iterations == r_st.iterations
    assert abs(r_lv.cost - r_st.cost) <= 1e-9 * r_st.cost
    for a, b in zip(p_lv, p_st):
        if a is not None:
            assert np.abs(a - b).max() <= 1e-7 * max(np.abs(b).max(), 1.0)


def _ulps(a, b):
    """Distance in units in the last place between float64 arrays of positive finite values."""
    ia = np.asarray(a, dtype=np.float64).view(np.int64)
    ib = np.asarray(b, dtype=np.float64).view(np.int64)
    return np.abs(ia - ib)


def test_pivot_reciprocals_are_accurate():
    """The tile factor's pivot reciprocal square root (the hardware approximation refined by one
    third-order Householder step) against an extended-precision host value and beside CUDA's rsqrt(),
    over positive pivots from 1e-300 to 1e300: within 2 ulp (CUDA's rsqrt() measured within 1)."""
    rng = np.random.default_rng(11)
    x = np.concatenate([10.0 ** rng.uniform(-300, 300, 20000), [1.0, 2.0, 0.5, 3.0, 1e-300, 1e300],
                        np.nextafter(1.0, 2.0) * np.arange(1, 100)])
    out = capi.check_pivot_reciprocals(x)
    rsqrt_host = (1 / np.sqrt(x.astype(np.longdouble))).astype(np.float64)
    ours, cuda = _ulps(out[:, 0], rsqrt_host), _ulps(out[:, 1], rsqrt_host)
    print(f"rsqrt_nr: max {ours.max()} ulp ({np.mean(ours > 0):.1%} not exact); CUDA rsqrt(): max {cuda.max()} ulp")
    assert ours.max() <= 2
    assert cuda.max() <= 2
