"""Seeded synthetic bundle-adjustment scenes.

The reference ships no data set for its bundle adjuster, so every workload is generated here
from a seed.  Each generator returns a :class:`Scene` whose arrays follow the layout of the
C-ABI (``include/v3dba.h``): row-major doubles, point-major observation order as produced by
the reference's ``BundlePointStructure`` (V3D/include/Geometry/v3d_mviewutilities.h:132-163),
0-based ``view`` / ``point`` indices.

Workloads:
  * :func:`circle_scene`    -- 20 pinhole cameras on a circle, 2,000 points, ~8k observations
  * :func:`sequence_scene`  -- 200-camera forward sequence with shared distorted intrinsics,
                               50,000 points, tracks of 3-12 consecutive views, 2% outliers
  * :func:`triplet_batch`   -- thousands of independent 3-camera problems of uneven size
  * :func:`cluster_scene`   -- 2,000 cameras in 20 groups, 1M points, ~6M observations
  * :func:`stereo_rig_scene` -- a binocular rig along a path (StereoMetricBundleOptimizer)
  * :func:`rotation_graph`  -- view graphs for rotation averaging (refineConsistentRotations)
  * :func:`triplet_stage_batch` -- triplets with raw tracks for the triplet stage (triangulation,
                               filtering, adjustment)
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

MODEL_STD, MODEL_COMMON, MODEL_VARYING, MODEL_STEREO = 0, 1, 2, 3
FULL_BUNDLE_NO_ROTATIONS, FULL_BUNDLE_METRIC, FULL_BUNDLE_FOCAL_LENGTH = -1, 0, 1
FULL_BUNDLE_FOCAL_LENGTH_PP, FULL_BUNDLE_RADIAL, FULL_BUNDLE_RADIAL_TANGENTIAL = 2, 3, 4


def intrinsic_dim(mode: int) -> int:
    return {1: 1, 2: 3, 3: 5, 4: 7}.get(mode, 0)


@dataclasses.dataclass
class Scene:
    model: int
    mode: int
    inlier_threshold: float
    K: np.ndarray          # (N,3,3) per camera, or (3,3) shared for MODEL_COMMON
    R: np.ndarray          # (N,3,3)
    T: np.ndarray          # (N,3)
    X: np.ndarray          # (M,3)
    meas: np.ndarray       # (K,2)
    view: np.ndarray       # (K,) int32
    point: np.ndarray      # (K,) int32
    dist: np.ndarray | None = None   # (4,) shared or (N,4)
    name: str = ""
    # MODEL_STEREO: R / T are rig poses; the L fixed rig cameras and each observation's camera
    rig_K: np.ndarray | None = None  # (L,3,3)
    rig_R: np.ndarray | None = None  # (L,3,3)
    rig_T: np.ndarray | None = None  # (L,3)
    sub: np.ndarray | None = None    # (K,) int32

    @property
    def n_cams(self) -> int:
        return int(self.R.shape[0])

    @property
    def n_points(self) -> int:
        return int(self.X.shape[0])

    @property
    def n_obs(self) -> int:
        return int(self.view.shape[0])

    @property
    def dims(self) -> tuple[int, int]:
        dA = 6 + (intrinsic_dim(self.mode) if self.model == MODEL_VARYING else 0)
        dC = intrinsic_dim(self.mode) if self.model == MODEL_COMMON else 0
        return dA, dC

    def copy(self) -> "Scene":
        return dataclasses.replace(
            self, K=self.K.copy(), R=self.R.copy(), T=self.T.copy(), X=self.X.copy(),
            meas=self.meas.copy(), view=self.view.copy(), point=self.point.copy(),
            dist=None if self.dist is None else self.dist.copy())

    @property
    def n_rig(self) -> int:
        return 0 if self.rig_K is None else int(self.rig_K.shape[0])

    def params(self):
        """(K, R, T, dist, X) as contiguous float64 arrays (dist is a 1-element dummy for STD)."""
        dist = self.dist if self.dist is not None else np.zeros(1)
        return tuple(np.ascontiguousarray(a, dtype=np.float64) for a in (self.K, self.R, self.T, dist, self.X))

    def set_params(self, K, R, T, dist, X):
        self.K[...] = K
        self.R[...] = R
        self.T[...] = T
        self.X[...] = X
        if self.dist is not None:
            self.dist[...] = dist


# ---------------------------------------------------------------------------------------------
# geometry helpers (vectorized)

def rodrigues(omega: np.ndarray) -> np.ndarray:
    """Rotation matrices exp([w]_x) for omega of shape (...,3)."""
    omega = np.asarray(omega, dtype=np.float64)
    th = np.linalg.norm(omega, axis=-1)[..., None, None]
    Kx = np.zeros(omega.shape[:-1] + (3, 3))
    Kx[..., 0, 1], Kx[..., 0, 2] = -omega[..., 2], omega[..., 1]
    Kx[..., 1, 0], Kx[..., 1, 2] = omega[..., 2], -omega[..., 0]
    Kx[..., 2, 0], Kx[..., 2, 1] = -omega[..., 1], omega[..., 0]
    safe = np.where(th > 1e-12, th, 1.0)
    c1 = np.where(th > 1e-12, np.sin(safe) / safe, 1.0)
    c2 = np.where(th > 1e-12, (1 - np.cos(safe)) / safe ** 2, 0.5)
    I = np.broadcast_to(np.eye(3), Kx.shape)
    return I + c1 * Kx + c2 * (Kx @ Kx)


def look_at(center: np.ndarray, target: np.ndarray, up: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """World->camera (R, T) for cameras at ``center`` (N,3) looking at ``target`` (N,3)."""
    z = target - center
    z /= np.linalg.norm(z, axis=-1, keepdims=True)
    x = np.cross(z, up)
    x /= np.linalg.norm(x, axis=-1, keepdims=True)
    y = np.cross(z, x)
    R = np.stack([x, y, z], axis=-2)
    T = -np.einsum("nij,nj->ni", R, center)
    return R, T


def random_unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def project_pinhole(K, R, T, X):
    """K(RX+T) dehomogenised; K,R,T broadcast against X (...,3)."""
    XX = np.einsum("...ij,...j->...i", R, X) + T
    h = np.einsum("...ij,...j->...i", K, XX)
    return h[..., :2] / h[..., 2:3], XX[..., 2]


def distort(dist, u):
    k1, k2, p1, p2 = dist[..., 0:1], dist[..., 1:2], dist[..., 2:3], dist[..., 3:4]
    x, y = u[..., 0:1], u[..., 1:2]
    r2 = x * x + y * y
    kr = 1 + k1 * r2 + k2 * r2 * r2
    xd = kr * x + 2 * p1 * x * y + p2 * (r2 + 2 * x * x)
    yd = kr * y + 2 * p2 * x * y + p1 * (r2 + 2 * y * y)
    return np.concatenate([xd, yd], axis=-1)


def project_distorted(K, R, T, dist, X):
    XX = np.einsum("...ij,...j->...i", R, X) + T
    u = XX[..., :2] / XX[..., 2:3]
    d = distort(dist, u)
    q0 = K[..., 0, 0] * d[..., 0] + K[..., 0, 1] * d[..., 1] + K[..., 0, 2]
    q1 = K[..., 1, 1] * d[..., 1] + K[..., 1, 2]
    return np.stack([q0, q1], axis=-1), XX[..., 2]


def _intrinsics(f, cx, cy):
    K = np.eye(3)
    K[0, 0] = K[1, 1] = f
    K[0, 2], K[1, 2] = cx, cy
    return K


def _perturb_cameras(rng, R, T, rot_rad, trans):
    n = R.shape[0]
    axis = random_unit(rng, n)
    dR = rodrigues(axis * rot_rad)
    return dR @ R, T + rng.normal(scale=trans, size=T.shape)


# ---------------------------------------------------------------------------------------------

def circle_scene(n_cams=20, n_points=2000, obs_per_point=4, seed=0, noise_px=0.5,
                 rot_perturb=0.02, trans_perturb=0.05, point_perturb=0.05,
                 inlier_threshold=1e6) -> Scene:
    """Plain metric BA: pinhole cameras (f=1000, pp (320,240), 640x480) on a circle of radius 10
    looking at the origin, points uniform in a cube of side 4, each seen by ``obs_per_point``
    random cameras in which it projects inside the image, N(0, noise_px) pixel noise, cameras
    perturbed by ``rot_perturb`` rad / N(0, trans_perturb) and points by N(0, point_perturb).
    Model: StdMetricBundleOptimizer; ``inlier_threshold`` 1e6 px makes it plain least squares."""
    rng = np.random.default_rng(seed)
    ang = 2 * np.pi * np.arange(n_cams) / n_cams
    centers = np.stack([10 * np.cos(ang), 10 * np.sin(ang), np.zeros(n_cams)], axis=1)
    R, T = look_at(centers, np.zeros_like(centers), np.array([0.0, 0.0, 1.0]))
    K = np.broadcast_to(_intrinsics(1000.0, 320.0, 240.0), (n_cams, 3, 3)).copy()
    X = rng.uniform(-2.0, 2.0, size=(n_points, 3))

    q, z = project_pinhole(K[None], R[None], T[None], X[:, None, :])      # (M,N,2)
    vis = (z > 0) & (q[..., 0] >= 0) & (q[..., 0] < 640) & (q[..., 1] >= 0) & (q[..., 1] < 480)
    views, points, meas = [], [], []
    keep = []
    for j in range(n_points):
        cand = np.flatnonzero(vis[j])
        if cand.size < 2:
            continue
        sel = np.sort(rng.choice(cand, size=min(obs_per_point, cand.size), replace=False))
        for i in sel:
            views.append(i)
            points.append(len(keep))
            meas.append(q[j, i] + rng.normal(scale=noise_px, size=2))
        keep.append(j)
    X = X[keep]
    R0, T0 = _perturb_cameras(rng, R, T, rot_perturb, trans_perturb)
    X0 = X + rng.normal(scale=point_perturb, size=X.shape)
    return Scene(MODEL_STD, FULL_BUNDLE_METRIC, inlier_threshold, K, R0, T0, X0,
                 np.asarray(meas, dtype=np.float64), np.asarray(views, dtype=np.int32),
                 np.asarray(points, dtype=np.int32), None, name=f"circle{n_cams}x{len(keep)}")


def sequence_scene(n_cams=200, n_points=50000, min_track=3, max_track=12, seed=0, noise_px=1.0,
                   outlier_frac=0.02, inlier_threshold=1.0, mode=FULL_BUNDLE_RADIAL_TANGENTIAL,
                   rot_perturb=0.005, trans_perturb=0.01, point_perturb=0.02,
                   f_init_scale=1.01) -> Scene:
    """Distortion BA: ``n_cams`` cameras along a forward-moving path sharing intrinsics
    (f=800, pp (320,240), 640x480, k1=-0.1, k2=0.01, p1=p2=1e-3), points in a corridor, each
    seen by a track of U{min_track..max_track} consecutive views where it projects in-image,
    N(0, noise_px) noise, ``outlier_frac`` of observations replaced by uniform pixels.
    Initial estimates: perturbed poses and points, f scaled by ``f_init_scale``, zero
    distortion.  Model: CommonInternalsMetricBundleOptimizer(``mode``), Huber threshold 1 px."""
    rng = np.random.default_rng(seed)
    max_track = min(max_track, n_cams)
    min_track = min(min_track, max_track)
    W_, H_ = 640.0, 480.0
    K_true = _intrinsics(800.0, 320.0, 240.0)
    dist_true = np.array([-0.1, 0.01, 1e-3, 1e-3])
    s = np.arange(n_cams, dtype=np.float64)
    centers = np.stack([0.4 * np.sin(s / 17.0), 0.15 * np.sin(s / 11.0), 0.25 * s], axis=1)
    yaw = 0.05 * np.sin(s / 23.0)
    pitch = 0.03 * np.sin(s / 29.0)
    R = rodrigues(np.stack([pitch, yaw, np.zeros(n_cams)], axis=1))
    T = -np.einsum("nij,nj->ni", R, centers)

    lengths = rng.integers(min_track, max_track + 1, size=n_points)
    starts = np.floor(rng.uniform(0, 1, size=n_points) * (n_cams - lengths + 1)).astype(np.int64)
    X = np.empty((n_points, 3))
    todo = np.arange(n_points)
    for _ in range(64):
        if todo.size == 0:
            break
        last = starts[todo] + lengths[todo] - 1
        depth = rng.uniform(1.5, 6.0, size=todo.size)
        cand = np.stack([rng.uniform(-0.3, 0.3, size=todo.size) * depth,
                         rng.uniform(-0.22, 0.22, size=todo.size) * depth, depth], axis=1)
        # place relative to the last camera of the track, in its camera frame
        Xw = np.einsum("nji,nj->ni", R[last], cand - T[last])
        ok = np.ones(todo.size, dtype=bool)
        for t in range(max_track):
            active = t < lengths[todo]
            cams = np.where(active, starts[todo] + t, 0)
            q, z = project_distorted(K_true, R[cams], T[cams], dist_true, Xw)
            inside = (z > 0.5) & (q[:, 0] >= 0) & (q[:, 0] < W_) & (q[:, 1] >= 0) & (q[:, 1] < H_)
            ok &= inside | ~active
        X[todo[ok]] = Xw[ok]
        todo = todo[~ok]
    if todo.size:
        keep = np.setdiff1d(np.arange(n_points), todo)
        X, lengths, starts = X[keep], lengths[keep], starts[keep]
    n_points = X.shape[0]

    point = np.repeat(np.arange(n_points, dtype=np.int32), lengths)
    offs = np.arange(point.size) - np.repeat(np.cumsum(lengths) - lengths, lengths)
    view = (np.repeat(starts, lengths) + offs).astype(np.int32)
    q, _ = project_distorted(K_true, R[view], T[view], dist_true, X[point])
    meas = q + rng.normal(scale=noise_px, size=q.shape)
    out = rng.uniform(size=point.size) < outlier_frac
    meas[out] = np.stack([rng.uniform(0, W_, size=out.sum()), rng.uniform(0, H_, size=out.sum())], axis=1)

    R0, T0 = _perturb_cameras(rng, R, T, rot_perturb, trans_perturb)
    X0 = X + rng.normal(scale=point_perturb, size=X.shape)
    K0 = K_true.copy()
    K0[0, 0] *= f_init_scale
    K0[1, 1] *= f_init_scale
    return Scene(MODEL_COMMON, mode, inlier_threshold, K0, R0, T0, X0, meas, view, point,
                 np.zeros(4), name=f"sequence{n_cams}x{n_points}")


def triplet_batch(n_triplets=4096, min_points=50, max_points=800, seed=0, noise_px=0.5,
                  inlier_threshold=1.0) -> list[Scene]:
    """Independent 3-camera problems: U{min_points..max_points} points each seen in all three
    views, baselines U[0.5, 2], convergence angles U[5, 30] degrees, f=1000, pp (320,240),
    N(0, noise_px) noise; initial poses and points perturbed.  Model: StdMetricBundleOptimizer
    (the reference's triplet stage uses inlier threshold 1 px and 5 iterations)."""
    rng = np.random.default_rng(seed)
    K = _intrinsics(1000.0, 320.0, 240.0)
    out = []
    for t in range(n_triplets):
        m = int(rng.integers(min_points, max_points + 1))
        b = rng.uniform(0.5, 2.0)
        alpha = np.deg2rad(rng.uniform(5.0, 30.0))
        D = b / (2 * np.sin(alpha / 2))
        ang = np.array([-alpha, 0.0, alpha])
        centers = np.stack([D * np.sin(ang), np.zeros(3), D - D * np.cos(ang)], axis=1)
        target = np.broadcast_to(np.array([0.0, 0.0, D]), (3, 3)).copy()
        R, T = look_at(centers, target, np.array([0.0, -1.0, 0.0]))
        rad = 0.18 * D
        X = np.array([0.0, 0.0, D]) + rng.uniform(-rad, rad, size=(m, 3))
        q, _ = project_pinhole(K[None], R[None], T[None], X[:, None, :])  # (m,3,2)
        meas = (q + rng.normal(scale=noise_px, size=q.shape)).reshape(-1, 2)
        view = np.tile(np.arange(3, dtype=np.int32), m)
        point = np.repeat(np.arange(m, dtype=np.int32), 3)
        R0, T0 = _perturb_cameras(rng, R, T, 0.01, 0.02 * b)
        X0 = X + rng.normal(scale=0.01 * D, size=X.shape)
        Ks = np.broadcast_to(K, (3, 3, 3)).copy()
        out.append(Scene(MODEL_STD, FULL_BUNDLE_METRIC, inlier_threshold, Ks, R0, T0, X0,
                         meas, view, point, None, name=f"triplet{t}"))
    return out


def cluster_scene(n_groups=20, cams_per_group=100, n_points=1_000_000, seed=0, noise_px=1.0,
                  cross_frac=0.05, mean_track=6.0, min_track=2, inlier_threshold=1e6) -> Scene:
    """Large scene: ``n_groups`` clusters of ``cams_per_group`` cameras on circles of radius 8
    around group centres spaced 12 apart; each point is seen by a geometric track (mean
    ``mean_track``, min ``min_track``) of cameras of its group, and ``cross_frac`` of the points
    sit between two neighbouring groups and are seen from both (the sparse inter-group
    co-visibility).  f=1000, pp (320,240), 640x480, N(0, noise_px) noise.  Model: Std."""
    rng = np.random.default_rng(seed)
    n_cams = n_groups * cams_per_group
    K1 = _intrinsics(1000.0, 320.0, 240.0)
    gc = np.stack([12.0 * np.arange(n_groups), np.zeros(n_groups), np.zeros(n_groups)], axis=1)
    ang = 2 * np.pi * rng.uniform(size=n_cams)
    elev = rng.uniform(-0.3, 0.3, size=n_cams)
    grp = np.repeat(np.arange(n_groups), cams_per_group)
    centers = gc[grp] + 8.0 * np.stack([np.cos(ang) * np.cos(elev), np.sin(ang) * np.cos(elev), np.sin(elev)], axis=1)
    look = gc[grp] + rng.normal(scale=0.5, size=(n_cams, 3))
    R, T = look_at(centers, look, np.array([0.0, 0.0, 1.0]))
    K = np.broadcast_to(K1, (n_cams, 3, 3)).copy()

    p = 1.0 / (mean_track - min_track + 1)
    lengths = min_track - 1 + rng.geometric(p, size=n_points)
    cross = (rng.uniform(size=n_points) < cross_frac) & (n_groups > 1)
    pg = rng.integers(0, n_groups - 1 if n_groups > 1 else 1, size=n_points)
    base = gc[pg].copy()
    base[cross, 0] += 6.0
    X = base + rng.uniform(-2.5, 2.5, size=(n_points, 3))

    views_l, pts_l = [], []
    chunk = 20000
    kept = np.zeros(n_points, dtype=bool)
    ncand = 48
    big = np.iinfo(np.int64).max
    for c0 in range(0, n_points, chunk):
        idx = np.arange(c0, min(c0 + chunk, n_points))
        # candidate cameras: the point's group, plus the next group for cross points
        cand_g = np.stack([pg[idx], np.where(cross[idx], pg[idx] + 1, pg[idx])], axis=1)
        cams = (cand_g[:, rng.integers(0, 2, size=ncand)] * cams_per_group
                + rng.integers(0, cams_per_group, size=(idx.size, ncand)))
        q, z = project_pinhole(K[cams], R[cams], T[cams], X[idx][:, None, :])
        vis = (z > 0.5) & (q[..., 0] >= 0) & (q[..., 0] < 640) & (q[..., 1] >= 0) & (q[..., 1] < 480)
        # distinct visible candidates, then a random subset of the track length, sorted
        o = np.argsort(cams, axis=1, kind="stable")
        cs = np.take_along_axis(cams, o, 1)
        vs = np.take_along_axis(vis, o, 1)
        vs[:, 1:] &= cs[:, 1:] != cs[:, :-1]
        cnt = vs.sum(axis=1)
        ok = cnt >= min_track
        L = np.where(ok, np.minimum(lengths[idx], cnt), 0)
        key = np.where(vs, rng.uniform(size=vs.shape), 2.0)
        pick = np.take_along_axis(cs, np.argsort(key, axis=1), 1)
        take = np.arange(ncand)[None, :] < L[:, None]
        sel = np.sort(np.where(take, pick, big), axis=1)
        take = np.sort(take, axis=1)[:, ::-1]
        views_l.append(sel[take])
        pts_l.append(np.repeat(idx, L))
        kept[idx[ok]] = True
    views, pts = np.concatenate(views_l), np.concatenate(pts_l)
    remap = -np.ones(n_points, dtype=np.int64)
    remap[kept] = np.arange(int(kept.sum()))
    X = X[kept]
    point = remap[pts].astype(np.int32)
    view = views.astype(np.int32)
    q, _ = project_pinhole(K[view], R[view], T[view], X[point])
    meas = q + rng.normal(scale=noise_px, size=q.shape)
    R0, T0 = _perturb_cameras(rng, R, T, 0.005, 0.02)
    X0 = X + rng.normal(scale=0.02, size=X.shape)
    return Scene(MODEL_STD, FULL_BUNDLE_METRIC, inlier_threshold, K, R0, T0, X0, meas, view,
                 point, None, name=f"cluster{n_cams}x{X.shape[0]}")


def scaled_sequence_scene(n_cams=20, n_points=2000, seed=0, **kw) -> Scene:
    """A small twin of :func:`sequence_scene` for parity tests."""
    return sequence_scene(n_cams=n_cams, n_points=n_points, seed=seed, **kw)


def varying_scene(n_cams=12, n_points=800, seed=0, mode=FULL_BUNDLE_RADIAL_TANGENTIAL) -> Scene:
    """Per-camera intrinsics and distortion (VaryingInternalsMetricBundleOptimizer), built from a
    short forward sequence whose cameras each get their own slightly different K and distortion."""
    sc = sequence_scene(n_cams=n_cams, n_points=n_points, seed=seed, outlier_frac=0.0,
                        min_track=3, max_track=min(8, n_cams), mode=mode)
    rng = np.random.default_rng(seed + 1000)
    N = sc.n_cams
    K = np.broadcast_to(sc.K, (N, 3, 3)).copy()
    K[:, 0, 0] *= 1 + rng.normal(scale=0.003, size=N)
    K[:, 1, 1] = K[:, 0, 0] * 1.001
    dist = np.zeros((N, 4))
    return Scene(MODEL_VARYING, mode, 1.0, K, sc.R, sc.T, sc.X, sc.meas, sc.view, sc.point, dist,
                 name=f"varying{N}x{sc.n_points}")


@dataclasses.dataclass
class RotationGraph:
    """Input of refineConsistentRotations: relative rotations R_ij ~ R_j R_i^T of view pairs
    (i, j) and initial absolute rotations.  ``rel`` (n_pairs, 3, 3), ``pairs`` (n_pairs, 2) int32,
    ``R0`` (n_views, 3, 3), ``R_true`` (n_views, 3, 3) the noise-free rotations."""
    rel: np.ndarray
    pairs: np.ndarray
    R0: np.ndarray
    R_true: np.ndarray
    name: str = "rotations"

    @property
    def n_views(self) -> int:
        return int(self.R0.shape[0])

    @property
    def n_pairs(self) -> int:
        return int(self.pairs.shape[0])


def rotation_graph(n_views=2000, n_pairs=40000, window=5, noise_deg=1.0, init_deg=5.0, outlier_frac=0.0,
                   seed=0) -> RotationGraph:
    """A view graph as an SfM pipeline produces it: every view paired with its ``window`` next
    views along the capture order, the remaining pairs drawn uniformly among all views (loop
    closures), in random order.  Relative rotations carry ``noise_deg`` of rotation noise (a
    fraction ``outlier_frac`` of them are random rotations); the initial rotations are the true
    ones perturbed by ``init_deg``."""
    rng = np.random.default_rng(seed)
    ax = random_unit(rng, n_views)
    R_true = rodrigues(ax * rng.uniform(0.0, math.pi, size=(n_views, 1)))
    seq = [(i, i + d) for d in range(1, window + 1) for i in range(n_views - d)]
    have = set(seq)
    pairs = list(seq[:n_pairs])
    while len(pairs) < n_pairs and len(have) < n_views * (n_views - 1) // 2:
        i, j = (int(v) for v in rng.integers(0, n_views, size=2))
        if i == j:
            continue
        i, j = min(i, j), max(i, j)
        if (i, j) in have:
            continue
        have.add((i, j))
        pairs.append((i, j))
    pairs = np.array(pairs, dtype=np.int32).reshape(-1, 2)
    pairs = pairs[rng.permutation(len(pairs))]
    flip = rng.random(len(pairs)) < 0.5     # either orientation of a pair
    pairs[flip] = pairs[flip][:, ::-1]
    i, j = pairs[:, 0], pairs[:, 1]
    rel = R_true[j] @ np.transpose(R_true[i], (0, 2, 1))
    noise = rodrigues(rng.normal(scale=math.radians(noise_deg), size=(len(pairs), 3)))
    rel = noise @ rel
    n_out = int(round(outlier_frac * len(pairs)))
    if n_out:
        sel = rng.choice(len(pairs), size=n_out, replace=False)
        rel[sel] = rodrigues(random_unit(rng, n_out) * rng.uniform(0.0, math.pi, size=(n_out, 1)))
    R0 = R_true @ rodrigues(rng.normal(scale=math.radians(init_deg), size=(n_views, 3)))
    return RotationGraph(np.ascontiguousarray(rel), np.ascontiguousarray(pairs), np.ascontiguousarray(R0),
                         R_true, name=f"rotations{n_views}x{len(pairs)}")


def stereo_rig_scene(n_poses=30, n_points=3000, baseline=0.3, seed=0, noise_px=0.5, outlier_frac=0.0,
                     inlier_threshold=2.0, rot_perturb=0.01, trans_perturb=0.02, point_perturb=0.05,
                     window=4) -> Scene:
    """Rig BA (StereoMetricBundleOptimizer): a binocular rig (camera 0 at the rig origin, camera 1
    ``baseline`` to its right and toed in by 2 degrees, slightly different intrinsics, 640x480)
    moving forward along a gently curving path; points in a corridor ahead; every point is seen
    from up to ``window`` consecutive rig poses, by each rig camera in which it projects inside
    the image (N(0, noise_px) pixel noise, ``outlier_frac`` gross outliers).  The poses are
    perturbed by ``rot_perturb`` rad / N(0, trans_perturb) and the points by N(0, point_perturb);
    Huber threshold ``inlier_threshold`` px."""
    rng = np.random.default_rng(seed)
    rig_K = np.stack([_intrinsics(700.0, 320.0, 240.0), _intrinsics(705.0, 318.0, 242.0)])
    rig_R = np.stack([np.eye(3), rodrigues(np.array([0.0, math.radians(-2.0), 0.0]))])
    rig_T = np.stack([np.zeros(3), -rig_R[1] @ np.array([baseline, 0.0, 0.0])])
    # rig centres along z with a slow sway; the rig looks along +z (world -> rig: Y = R X + T)
    t = np.arange(n_poses, dtype=np.float64)
    centers = np.stack([0.5 * np.sin(0.15 * t), 0.1 * np.cos(0.2 * t), 0.8 * t], axis=1)
    yaw = 0.05 * np.sin(0.1 * t)
    R = rodrigues(np.stack([np.zeros(n_poses), yaw, np.zeros(n_poses)], axis=1))
    T = -np.einsum("nij,nj->ni", R, centers)
    X = np.stack([rng.uniform(-4, 4, n_points), rng.uniform(-3, 3, n_points),
                  rng.uniform(3.0, 0.8 * n_poses + 12.0, n_points)], axis=1)
    views, points, subs, meas, keep = [], [], [], [], []
    for j in range(n_points):
        first = int(np.clip(np.floor((X[j, 2] - 12.0) / 0.8), 0, n_poses - 1))
        obs = []
        for i in range(first, min(n_poses, first + window)):
            Y = R[i] @ X[j] + T[i]
            for l in range(2):
                Z = rig_R[l] @ Y + rig_T[l]
                if Z[2] <= 0.5:
                    continue
                h = rig_K[l] @ Z
                q = h[:2] / h[2]
                if 0 <= q[0] < 640 and 0 <= q[1] < 480:
                    obs.append((i, l, q))
        if len(obs) < 3:
            continue
        for i, l, q in obs:
            views.append(i)
            points.append(len(keep))
            subs.append(l)
            meas.append(q + rng.normal(scale=noise_px, size=2))
        keep.append(j)
    meas = np.asarray(meas, dtype=np.float64)
    n_out = int(round(outlier_frac * len(meas)))
    if n_out:
        sel = rng.choice(len(meas), size=n_out, replace=False)
        meas[sel] += rng.normal(scale=30.0, size=(n_out, 2))
    X = X[keep]
    R0, T0 = _perturb_cameras(rng, R, T, rot_perturb, trans_perturb)
    X0 = X + rng.normal(scale=point_perturb, size=X.shape)
    return Scene(MODEL_STEREO, FULL_BUNDLE_METRIC, inlier_threshold, np.zeros((1, 3, 3)), R0, T0, X0, meas,
                 np.asarray(views, dtype=np.int32), np.asarray(points, dtype=np.int32), None,
                 name=f"stereo{n_poses}x{len(keep)}", rig_K=rig_K, rig_R=rig_R, rig_T=rig_T,
                 sub=np.asarray(subs, dtype=np.int32))


@dataclasses.dataclass
class TripletTracks:
    """One triplet as the triplet stage receives it after connectTracks: the three cameras (K = I,
    world -> camera R (3,3,3), T (3,3)), each view's average focal length (3,), and the tracks:
    ``track_ptr`` (n+1,) int32 into ``view`` (int32) / ``pos`` (float32, normalised coordinates)."""
    R: np.ndarray
    T: np.ndarray
    focal: np.ndarray
    track_ptr: np.ndarray
    view: np.ndarray
    pos: np.ndarray

    @property
    def n_tracks(self) -> int:
        return int(self.track_ptr.shape[0] - 1)


def triplet_stage_batch(n_triplets=4096, min_tracks=30, max_tracks=800, seed=0, noise_px=0.3,
                        outlier_frac=0.1, two_view_frac=0.05, pose_rot_deg=0.01, pose_trans=0.0005,
                        bad_frac=0.05, bad_outlier_frac=0.7) -> list[TripletTracks]:
    """Triplets for the triplet stage: U{min_tracks..max_tracks} tracks each, geometry as in
    :func:`triplet_batch` but in normalised coordinates (focal lengths U[700, 1200] px per view),
    N(0, noise_px) pixel noise, a fraction ``outlier_frac`` of measurements replaced by wrong
    matches 5-40 px away, ``two_view_frac`` of the tracks seen in two views only, and the
    relative-pose error of the cameras (``pose_rot_deg``, ``pose_trans`` of the baseline).  A
    fraction ``bad_frac`` of the triplets get ``bad_outlier_frac`` wrong matches (the stage must
    drop them)."""
    rng = np.random.default_rng(seed)
    out = []
    for t in range(n_triplets):
        m = int(rng.integers(min_tracks, max_tracks + 1))
        b = rng.uniform(0.5, 2.0)
        alpha = np.deg2rad(rng.uniform(5.0, 30.0))
        D = b / (2 * np.sin(alpha / 2))
        ang = np.array([-alpha, 0.0, alpha])
        centers = np.stack([D * np.sin(ang), np.zeros(3), D - D * np.cos(ang)], axis=1)
        target = np.broadcast_to(np.array([0.0, 0.0, D]), (3, 3)).copy()
        R, T = look_at(centers, target, np.array([0.0, -1.0, 0.0]))
        focal = rng.uniform(700.0, 1200.0, size=3)
        X = np.array([0.0, 0.0, D]) + rng.uniform(-0.18 * D, 0.18 * D, size=(m, 3))
        Y = np.einsum("vij,mj->mvi", R, X) + T[None]
        q = Y[..., :2] / Y[..., 2:3]                                            # (m,3,2)
        q = q + rng.normal(size=q.shape) * (noise_px / focal)[None, :, None]
        frac = bad_outlier_frac if rng.random() < bad_frac else outlier_frac
        bad = rng.random((m, 3)) < frac
        disp = rng.uniform(5.0, 40.0, size=(m, 3)) / focal[None, :]
        phi = rng.uniform(0, 2 * np.pi, size=(m, 3))
        q[..., 0] += np.where(bad, disp * np.cos(phi), 0.0)
        q[..., 1] += np.where(bad, disp * np.sin(phi), 0.0)
        keep = np.ones((m, 3), dtype=bool)
        two = rng.random(m) < two_view_frac
        keep[two, rng.integers(0, 3, size=int(two.sum()))] = False
        counts = keep.sum(axis=1)
        track_ptr = np.zeros(m + 1, dtype=np.int32)
        track_ptr[1:] = np.cumsum(counts)
        view = np.nonzero(keep)[1].astype(np.int32)
        pos = q[keep].astype(np.float32)
        R0, T0 = _perturb_cameras(rng, R, T, np.deg2rad(pose_rot_deg), pose_trans * b)
        out.append(TripletTracks(np.ascontiguousarray(R0), np.ascontiguousarray(T0), focal, track_ptr, view,
                                 np.ascontiguousarray(pos.reshape(-1, 2))))
    return out

