"""Shared helpers of the test suite (fixture loading, scene construction, comparisons)."""
import glob
import os

import numpy as np

from v3dsfmtoolkit_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_names():
    return sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    sc = scenes.Scene(int(g["model"]), int(g["mode"]), float(g["inlier_threshold"]), g["K0"].copy(),
                      g["R0"].copy(), g["T0"].copy(), g["X0"].copy(), g["meas"].copy(), g["view"].copy(),
                      g["point"].copy(), g["dist0"].copy() if g["dist0"].size else None, name=name)
    if "rig_K" in g.files:
        sc.rig_K, sc.rig_R, sc.rig_T, sc.sub = g["rig_K"].copy(), g["rig_R"].copy(), g["rig_T"].copy(), g["sub"].copy()
    return sc, g


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def param_rel(pa, pb):
    """max relative difference over K, R, T, X (and distortion when present)."""
    out = 0.0
    for a, b in zip(pa, pb):
        a, b = np.asarray(a), np.asarray(b)
        if a.size == 0 or b.size == 0:
            continue
        out = max(out, rel(a, b))
    return out


def similarity_align(R, T, X, R_ref, T_ref, X_ref):
    """Moves the reconstruction (R, T, X) by the 7-DoF similarity (scale s, rotation Q,
    translation t) that best maps its points onto X_ref in the least-squares sense (Umeyama's
    closed form), and returns the moved (R', T', X'): X' = s Q X + t, R_i' = R_i Q^T,
    T_i' = s T_i - R_i' t.  Every projection K (R_i X_j + T_i) is unchanged (up to the scale s of
    the homogeneous point), so a bundle adjustment cannot tell the two apart: this is the gauge
    freedom of metric BA, and two solvers that reach the same minimum may differ by it."""
    X, X_ref = np.asarray(X, np.float64), np.asarray(X_ref, np.float64)
    mu, mu_ref = X.mean(axis=0), X_ref.mean(axis=0)
    A, B = X - mu, X_ref - mu_ref
    U, sig, Vt = np.linalg.svd(B.T @ A / len(X))
    D = np.eye(3)
    if np.linalg.det(U) * np.linalg.det(Vt) < 0:
        D[2, 2] = -1.0
    Q = U @ D @ Vt
    s = float(np.trace(np.diag(sig) @ D) / (A * A).sum(axis=1).mean())
    t = mu_ref - s * Q @ mu
    Xa = s * X @ Q.T + t
    Ra = np.asarray(R, np.float64) @ Q.T
    Ta = s * np.asarray(T, np.float64) - np.einsum("nij,j->ni", Ra, t)
    return Ra, Ta, Xa


ROT_GOLDEN = os.path.join(GOLDEN, "rotations")


def rotation_golden_names():
    return sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(ROT_GOLDEN, "*.npz")))


def load_rotation_golden(name):
    """(RotationGraph, fixture) of a rotation-averaging fixture."""
    g = np.load(os.path.join(ROT_GOLDEN, name + ".npz"))
    graph = scenes.RotationGraph(g["rel"].copy(), g["pairs"].copy(), g["R0"].copy(), g["R"].copy(), name=name)
    return graph, g


def load_triplet_stage_golden():
    """(list of TripletTracks, list of the reference's per-triplet outputs) of
    tests/golden/triplets/stage.npz."""
    g = np.load(os.path.join(GOLDEN, "triplets", "stage.npz"))
    trips, outs = [], []
    tp, mo = g["tp_off"], g["m_off"]
    x0 = 0
    for i in range(len(g["verdict"])):
        ptr = g["track_ptr"][tp[i]:tp[i + 1]]
        n = len(ptr) - 1
        trips.append(scenes.TripletTracks(g["R"][i], g["T"][i], g["focal"][i], ptr, g["view"][mo[i]:mo[i + 1]],
                                          g["pos"][mo[i]:mo[i + 1]]))
        outs.append(dict(verdict=int(g["verdict"][i]), n_points=int(g["n_points"][i]), status=int(g["status"][i]),
                         iterations=int(g["iterations"][i]), cost=float(g["cost"][i]), R=g["R_out"][i],
                         T=g["T_out"][i], X=g["X_out"][x0:x0 + n], kept=g["kept"][mo[i]:mo[i + 1]]))
        x0 += n
    return trips, outs

