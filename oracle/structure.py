"""CPU restatement (numpy / Python) of the problem structure v3dba_create builds on the device --
test infrastructure only.

The reference derives the sparsity pattern of its full normal matrix on the host
(SparseLevenbergOptimizer::setupSparseJtJ, V3D/src/Math/v3d_optimization.cpp:301-554) from the
flat BundlePointStructure arrays (V3D/include/Geometry/v3d_mviewutilities.h:132-163); the GPU
build keeps, for the point-eliminated system, the orderings restated here:

  * o_orig: observations sorted by point, stable (the caller's order inside a track);
  * c_ptr / c_obs: each camera's observations in point-major order;
  * camera-pair blocks (i, l), i <= l, in (i, l) order, every camera with its diagonal block
    (empty when it has no observation), and per block its pairs (k, m) -- observation k of
    camera i and m of camera l of the same point -- ordered by k, then m.
"""
from __future__ import annotations

import numpy as np


def structure(n_cams, view, point):
    view = np.asarray(view, dtype=np.int64)
    point = np.asarray(point, dtype=np.int64)
    K = view.size
    o_orig = np.argsort(point, kind="stable")
    o_cam = view[o_orig]
    o_pt = point[o_orig]
    c_ptr = np.zeros(n_cams + 1, dtype=np.int64)
    np.add.at(c_ptr, o_cam + 1, 1)
    c_ptr = np.cumsum(c_ptr)
    c_obs = np.argsort(o_cam, kind="stable")
    # point tracks in point-major order
    starts = {}
    for k in range(K):
        starts.setdefault(int(o_pt[k]), []).append(k)
    b_i, b_l, b_ptr, pr_k, pr_m = [], [], [0], [], []
    for i in range(n_cams):
        per_l = {}
        for k in c_obs[c_ptr[i]:c_ptr[i + 1]]:
            for m in starts[int(o_pt[k])]:
                l = int(o_cam[m])
                if l >= i:
                    per_l.setdefault(l, []).append((int(k), m))
        per_l.setdefault(i, [])
        for l in sorted(per_l):
            for k, m in per_l[l]:
                pr_k.append(k)
                pr_m.append(m)
            b_i.append(i)
            b_l.append(l)
            b_ptr.append(len(pr_k))
    as32 = lambda a: np.asarray(a, dtype=np.int32)
    return {"o_orig": as32(o_orig), "c_ptr": as32(c_ptr), "c_obs": as32(c_obs), "b_i": as32(b_i), "b_l": as32(b_l),
            "b_ptr": as32(b_ptr), "pr_k": as32(pr_k), "pr_m": as32(pr_m)}
