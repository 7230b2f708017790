"""Small damped reduced camera systems for the learned-preconditioner tests, built on the CPU by
the oracle restatement (normal equations + Schur complement) from seeded scenes."""
from __future__ import annotations

import numpy as np

from v3dsfmtoolkit_b200 import scenes


def reduced_blocks(sc, lam_rel, params=None):
    """(n_cams, blk_i, blk_l, blocks, diag_index, S) of the damped reduced camera system of `sc`
    (6-parameter cameras) at lambda = lam_rel * max diagonal, blocks S_{i,l} for i <= l."""
    from oracle.bindings import Restatement
    R = Restatement()
    blk = R.normal_blocks(sc, params)
    mx = max(float(np.max(np.diagonal(blk["U"], axis1=1, axis2=2))),
             float(np.max(np.diagonal(blk["V"], axis1=1, axis2=2))))
    S, _, _, _ = R.reduced_system(sc, blk, lam_rel * mx)
    N = sc.n_cams
    bi, bl, bs, diag = [], [], [], {}
    for i in range(N):
        for l in range(i, N):
            B = S[6 * i:6 * i + 6, 6 * l:6 * l + 6]
            if i == l or np.any(B != 0.0):
                if i == l:
                    diag[i] = len(bi)
                bi.append(i)
                bl.append(l)
                bs.append(B.copy())
    return N, np.array(bi), np.array(bl), np.array(bs), np.array([diag[i] for i in range(N)]), S


def small_sequence(n_cams=10, seed=3):
    return scenes.sequence_scene(n_cams=n_cams, n_points=60 * n_cams, mode=scenes.FULL_BUNDLE_METRIC, seed=seed,
                                 outlier_frac=0.0)


def dense_pcg(S, b, apply, tol=1e-6, max_iter=5000):
    """Preconditioned CG on a dense matrix (FP64): iterations to |r| <= tol |b|."""
    x = np.zeros_like(b)
    r = b.copy()
    z = apply(r)
    p = z.copy()
    rz = r @ z
    b0 = np.linalg.norm(b)
    for it in range(1, max_iter + 1):
        q = S @ p
        a = rz / (p @ q)
        x += a * p
        r -= a * q
        if np.linalg.norm(r) <= tol * b0:
            return it
        z = apply(r)
        rz2 = r @ z
        p = z + (rz2 / rz) * p
        rz = rz2
    return max_iter


def converged_system(n_cams=60, seed=4, lam_rel=1e-10, iterations=20):
    """A sequence scene after `iterations` oracle LM iterations and its reduced system there."""
    from oracle.bindings import Restatement
    sc = scenes.sequence_scene(n_cams=n_cams, n_points=100 * n_cams, mode=scenes.FULL_BUNDLE_METRIC, seed=seed,
                               outlier_frac=0.0)
    params, _ = Restatement().minimize(sc, max_iterations=iterations)
    N, bi, bl, bs, diag, S = reduced_blocks(sc, lam_rel, params)
    R = np.asarray(params[1]).reshape(-1, 9)
    T = np.asarray(params[2]).reshape(-1, 3)
    return N, bi, bl, bs, diag, S, R, T
