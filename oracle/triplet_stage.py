"""TEST INFRASTRUCTURE ONLY: numpy restatement of the triplet stage around the triplet
adjustment (SfM/generate_triples/src/generate_triples.cpp:380-415), the checker of the GPU's
v3dba_triplet_stage.

* :func:`triangulate_linear` -- triangulateLinear (V3D/include/Geometry/v3d_mviewutilities.h:
  260-303): the 2K x 3 linear system of a track, solved by Householder QR as TNT's QR does it
  (V3D/include/Math/v3d_linear_tnt.h:1589-1629, solve :1734-1771), in the same operation order
  (Python floats are IEEE doubles; hypot is the C library's, called through ctypes, since
  Python's own math.hypot rounds differently).
* :func:`filter_track` -- filterTripleModel (generate_triples.cpp:44-81): the projection rounded
  to float, the float difference, float sum of squares and square root, times the view's focal
  length.
* :func:`stage` -- the survival tests (generate_triples.cpp:393-398) and the adjustment of the
  survivors (StdMetricBundleOptimizer, K = I) by the C restatement of the LM.

Only tests use this module.  It is pinned against the reference compiled from its sources
(tests/golden/triplets/stage.npz, tests/test_triplet_stage_oracle.py).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

_libm = ctypes.CDLL(None)
_libm.hypot.restype = ctypes.c_double
_libm.hypot.argtypes = [ctypes.c_double, ctypes.c_double]
_hypot = _libm.hypot


def _qr_least_squares(A, b):
    A = [list(map(float, row)) for row in A]
    x = [float(v) for v in b]
    m, n = len(A), 3
    rdiag = [0.0] * n
    for k in range(n):
        nrm = 0.0
        for i in range(k, m):
            nrm = _hypot(nrm, A[i][k])
        if nrm != 0.0:
            if A[k][k] < 0:
                nrm = -nrm
            for i in range(k, m):
                A[i][k] /= nrm
            A[k][k] += 1.0
            for j in range(k + 1, n):
                s = 0.0
                for i in range(k, m):
                    s += A[i][k] * A[i][j]
                s = -s / A[k][k]
                for i in range(k, m):
                    A[i][j] += s * A[i][k]
        rdiag[k] = -nrm
    if any(r == 0.0 for r in rdiag):
        return None
    for k in range(n):
        s = 0.0
        for i in range(k, m):
            s += A[i][k] * x[i]
        s = -s / A[k][k]
        for i in range(k, m):
            x[i] += s * A[i][k]
    for k in range(n - 1, -1, -1):
        x[k] /= rdiag[k]
        for i in range(k):
            x[i] -= x[k] * A[i][k]
    return np.array(x[:n])


def triangulate_linear(R, T, views, pos):
    """Point of one track: rows x P_2 - P_0, y P_2 - P_1 with P = [R | T] (K = I)."""
    A, b = [], []
    for v, (x, y) in zip(views, pos):
        x, y = float(np.float32(x)), float(np.float32(y))
        P = np.concatenate([R[v], T[v][:, None]], axis=1)
        A.append([x * P[2][c] - P[0][c] for c in range(3)])
        A.append([y * P[2][c] - P[1][c] for c in range(3)])
        b.append(P[0][3] - x * P[2][3])
        b.append(P[1][3] - y * P[2][3])
    if len(A) < 3:
        return np.full(3, np.nan)
    X = _qr_least_squares(A, b)
    return np.full(3, np.nan) if X is None else X


def filter_track(R, T, focal, views, pos, X, max_err):
    """Measurement survival flags of one track."""
    keep = []
    for v, (mx, my) in zip(views, pos):
        Rv, Tv = R[v], T[v]
        q = [Rv[r][0] * X[0] + Rv[r][1] * X[1] + Rv[r][2] * X[2] + Tv[r] for r in range(3)]
        px, py = np.float32(q[0] / q[2]), np.float32(q[1] / q[2])
        dx, dy = px - np.float32(mx), py - np.float32(my)
        n = np.float32(math.sqrt(float(dx * dx + dy * dy)))
        err = float(focal[v]) * float(n)
        keep.append(err < max_err)
    return np.array(keep, dtype=bool)


def stage(trip, max_reproj_error=1.0, min_points=50, min_point_ratio=0.5, inlier_threshold=1.0, tau=1e-3,
          max_iterations=5):
    """The restated stage on one TripletTracks: dict like the reference wrapper's."""
    from oracle.bindings import Restatement
    from v3dsfmtoolkit_b200 import scenes
    n = trip.n_tracks
    X = np.zeros((n, 3))
    kept = np.zeros(int(trip.track_ptr[-1]), dtype=np.uint8)
    surv = []
    for j in range(n):
        a, b = int(trip.track_ptr[j]), int(trip.track_ptr[j + 1])
        views, pos = trip.view[a:b], trip.pos[a:b]
        X[j] = triangulate_linear(trip.R, trip.T, views, pos)
        k = filter_track(trip.R, trip.T, trip.focal, views, pos, X[j], max_reproj_error)
        kept[a:b] = k
        if k.sum() >= 3:
            surv.append(j)
    verdict = 0
    if len(surv) < min_points:
        verdict = 1
    elif float(len(surv)) < min_point_ratio * n:
        verdict = 2
    out = dict(verdict=verdict, n_points=len(surv), status=0, iterations=0, cost=0.0, R=trip.R.copy(),
               T=trip.T.copy(), X=X, kept=kept)
    if verdict != 0:
        return out
    meas, view, point = [], [], []
    for q, j in enumerate(surv):
        a, b = int(trip.track_ptr[j]), int(trip.track_ptr[j + 1])
        for m in range(a, b):
            if kept[m]:
                meas.append([float(trip.pos[m, 0]), float(trip.pos[m, 1])])
                view.append(int(trip.view[m]))
                point.append(q)
    K = np.broadcast_to(np.eye(3), (3, 3, 3)).copy()
    sc = scenes.Scene(scenes.MODEL_STD, 0, inlier_threshold, K, trip.R.copy(), trip.T.copy(), X[surv].copy(),
                      np.array(meas), np.array(view, dtype=np.int32), np.array(point, dtype=np.int32), None)
    (_, R, T, _, Xs), info = Restatement().minimize(sc, tau=tau, max_iterations=max_iterations)
    X[surv] = Xs
    out.update(status=info["status"], iterations=info["iterations"],
               cost=float(info["trace_cost"][-1]) if len(info["trace_cost"]) else 0.0, R=R.reshape(3, 3, 3),
               T=T.reshape(3, 3), X=X)
    return out
