"""CPU restatement (numpy, FP64) of the learned PCG preconditioner -- test infrastructure only.

The reference has no iterative solver and no learned component (it factors the damped normal
equations with LDL^T, V3D/src/Math/v3d_optimization.cpp:1096-1145), so this module restates the
method of ``v3dsfmtoolkit_b200/csrc/precond_gnn.cu`` from its mathematics and is the check of
the CUDA kernels' features, network outputs, loss and weight gradients:

  * normalisation: C_i C_i^T = S_ii, F_e = C_b^-1 S_(b,a) C_a^-T for every edge a < b;
  * edge inputs [F, (F F)|pattern, (F F^T)|pattern], node inputs [1, log(1+deg), mean |F|^2,
    max |F|^2];
  * the message-passing network (3 edge updates, 2 node updates, hidden 64) and its analytic
    backward pass;
  * the probe loss |(I+E) S^ (I+E)^T z - z|^2 / (n m) with the same Rademacher probes (fmix32
    of MurmurHash3 over the entry index and the seed) and dL/dcoef;
  * the gauge basis Z of a camera set (the 7 similarity motions).

Parity of the preconditioned solve itself is checked against block-Jacobi PCG (oracle
``orc_pcg``) and the direct solve.  Nothing in the product path imports this file.
"""
from __future__ import annotations

import numpy as np

H, EDGE_IN, NODE_IN, OUT, PROBES = 64, 108, 4, 3, 16


def layout():
    """Offsets of the [W; b] blocks in the flat weight vector."""
    off, o = {}, 0
    for name, k, n in [("ein", EDGE_IN, H), ("nin", NODE_IN, H)] + [(f"m{l}", 3 * H, H) for l in range(3)] + \
            [(f"h{l}", 2 * H, H) for l in range(2)] + [("out", H, OUT)]:
        off[name] = (o, k, n)
        o += (k + 1) * n
    return off, o


LAYOUT, NWEIGHTS = layout()


def unpack(w):
    out = {}
    for name, (o, k, n) in LAYOUT.items():
        blk = np.asarray(w[o:o + (k + 1) * n], dtype=np.float64).reshape(k + 1, n)
        out[name] = (blk[:k], blk[k])
    return out


class Graph:
    def __init__(self, n_cams, blk_i, blk_l):
        self.N = int(n_cams)
        e = [(b, int(i), int(l)) for b, (i, l) in enumerate(zip(blk_i, blk_l)) if i != l]
        self.eblk = np.array([t[0] for t in e], dtype=np.int64)
        self.ea = np.array([t[1] for t in e], dtype=np.int64)
        self.eb = np.array([t[2] for t in e], dtype=np.int64)
        self.ne = len(e)
        self.lo = [[] for _ in range(self.N)]
        self.up = [[] for _ in range(self.N)]
        for k in range(self.ne):
            self.lo[self.eb[k]].append(k)
            self.up[self.ea[k]].append(k)
        self.lo = [sorted(x, key=lambda k: self.ea[k]) for x in self.lo]
        self.up = [sorted(x, key=lambda k: self.eb[k]) for x in self.up]
        self.deg = np.array([len(self.lo[i]) + len(self.up[i]) for i in range(self.N)])
        eid = {(int(a), int(b)): k for k, (a, b) in enumerate(zip(self.ea, self.eb))}
        self.tri = []   # per edge: list of (e1, e2, transposed)
        for k in range(self.ne):
            a, b = int(self.ea[k]), int(self.eb[k])
            t = []
            for m in range(a + 1, b):            # (F F)_(b,a): F_(b,m) F_(m,a)
                if (m, b) in eid and (a, m) in eid:
                    t.append((eid[(m, b)], eid[(a, m)], 0))
            for m in range(0, a):                # (F F^T)_(b,a): F_(b,m) F_(a,m)^T
                if (m, b) in eid and (m, a) in eid:
                    t.append((eid[(m, b)], eid[(m, a)], 1))
            self.tri.append(t)


def features(graph, blocks, diag_index):
    """blocks: (nb, 6, 6) S_{i,l} (rows of camera i); diag_index[i] = block id of (i, i)."""
    N = graph.N
    cinv = np.zeros((N, 6, 6))
    for i in range(N):
        L = np.linalg.cholesky(blocks[diag_index[i]])
        cinv[i] = np.linalg.inv(L)
    F = np.zeros((graph.ne, 6, 6))
    for k in range(graph.ne):
        a, b = graph.ea[k], graph.eb[k]
        F[k] = cinv[b] @ blocks[graph.eblk[k]].T @ cinv[a].T
    F2 = np.zeros_like(F)
    FFt = np.zeros_like(F)
    for k in range(graph.ne):
        for e1, e2, t in graph.tri[k]:
            if t == 0:
                F2[k] += F[e1] @ F[e2]
            else:
                FFt[k] += F[e1] @ F[e2].T
    xe = np.concatenate([F.reshape(-1, 36), F2.reshape(-1, 36), FFt.reshape(-1, 36)], axis=1)
    nrm = (F ** 2).sum(axis=(1, 2))
    xn = np.zeros((N, NODE_IN))
    for i in range(N):
        inc = graph.lo[i] + graph.up[i]
        s = nrm[inc]
        xn[i] = [1.0, np.log1p(len(inc)), s.mean() if len(inc) else 0.0, s.max() if len(inc) else 0.0]
    return xe, xn, cinv


def _mean_agg(graph, E):
    G = np.zeros((graph.N, E.shape[1]))
    for i in range(graph.N):
        inc = graph.lo[i] + graph.up[i]
        if inc:
            G[i] = E[inc].sum(axis=0) / len(inc)
    return G


def forward(w, graph, xe, xn):
    P = unpack(w)
    relu = lambda z: np.maximum(z, 0.0)
    c = {"E": [relu(xe @ P["ein"][0] + P["ein"][1])], "H": [relu(xn @ P["nin"][0] + P["nin"][1])],
         "A": [], "G": [], "C": [], "X": []}
    for l in range(3):
        E, Hn = c["E"][-1], c["H"][-1]
        X = np.concatenate([Hn[graph.eb], Hn[graph.ea], E], axis=1)
        A = relu(X @ P[f"m{l}"][0] + P[f"m{l}"][1])
        c["X"].append(X)
        c["A"].append(A)
        c["E"].append(E + A)
        if l < 2:
            G = _mean_agg(graph, c["E"][-1])
            Cn = relu(np.concatenate([Hn, G], axis=1) @ P[f"h{l}"][0] + P[f"h{l}"][1])
            c["G"].append(G)
            c["C"].append(Cn)
            c["H"].append(Hn + Cn)
    coef = c["E"][-1] @ P["out"][0] + P["out"][1]
    return coef, c


def probe_signs(seed, n):
    idx = np.arange(n, dtype=np.uint64)
    h = (idx * np.uint64(0x9E3779B1) + np.uint64(seed)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(16)
    h = (h * np.uint64(0x85EBCA6B)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(13)
    h = (h * np.uint64(0xC2B2AE35)) & np.uint64(0xFFFFFFFF)
    h ^= h >> np.uint64(16)
    return np.where(h & np.uint64(1), 1.0, -1.0)


def edge_blocks(xe, coef):
    c = 1.0 + coef
    return (-c[:, 0:1] * xe[:, :36] + c[:, 1:2] * xe[:, 36:72] + c[:, 2:3] * xe[:, 72:]).reshape(-1, 6, 6)


def _IEt(graph, E, v):
    out = v.copy()
    for k in range(graph.ne):
        out[graph.ea[k]] += E[k].T @ v[graph.eb[k]]
    return out


def _IE(graph, E, v):
    out = v.copy()
    for k in range(graph.ne):
        out[graph.eb[k]] += E[k] @ v[graph.ea[k]]
    return out


def _Shat(graph, F, v):
    out = v.copy()
    for k in range(graph.ne):
        a, b = graph.ea[k], graph.eb[k]
        out[b] += F[k] @ v[a]
        out[a] += F[k].T @ v[b]
    return out


def probe_loss(graph, xe, coef, seed):
    """Loss and dL/dcoef.  Probe vectors are (N, 6, PROBES)."""
    N = graph.N
    z = probe_signs(seed, N * 6 * PROBES).reshape(N, 6, PROBES)
    E = edge_blocks(xe, coef)
    F = xe[:, :36].reshape(-1, 6, 6)
    y = _IEt(graph, E, z)
    wv = _Shat(graph, F, y)
    p = _IE(graph, E, wv)
    scale = 1.0 / (N * 6 * PROBES)
    r = p - z
    loss = scale * float((r ** 2).sum())
    dp = 2.0 * scale * r
    dw = _IEt(graph, E, dp)
    dy = _Shat(graph, F, dw)
    dcoef = np.zeros((graph.ne, 3))
    for k in range(graph.ne):
        a, b = graph.ea[k], graph.eb[k]
        dE = dp[b] @ wv[a].T + z[b] @ dy[a].T
        dcoef[k, 0] = -(dE * xe[k, :36].reshape(6, 6)).sum()
        dcoef[k, 1] = (dE * xe[k, 36:72].reshape(6, 6)).sum()
        dcoef[k, 2] = (dE * xe[k, 72:].reshape(6, 6)).sum()
    return loss, dcoef


def backward(w, graph, xe, xn, cache, dcoef):
    P = unpack(w)
    grads = {}

    def put(name, X, D):
        grads[name] = np.concatenate([X.T @ D, D.sum(axis=0, keepdims=True)], axis=0)

    put("out", cache["E"][3], dcoef)
    dE = dcoef @ P["out"][0].T
    dH = np.zeros((graph.N, H))
    for l in (2, 1, 0):
        if l < 2:
            dZ = dH * (cache["C"][l] > 0)
            put(f"h{l}", np.concatenate([cache["H"][l], cache["G"][l]], axis=1), dZ)
            dX = dZ @ P[f"h{l}"][0].T
            dH = dH + dX[:, :H]
            dG = dX[:, H:]
            for k in range(graph.ne):
                a, b = graph.ea[k], graph.eb[k]
                dE[k] += dG[b] / graph.deg[b] + dG[a] / graph.deg[a]
        dZ = dE * (cache["A"][l] > 0)
        put(f"m{l}", cache["X"][l], dZ)
        dX = dZ @ P[f"m{l}"][0].T
        dE = dE + dX[:, 2 * H:]
        dHe = np.zeros((graph.N, H))
        np.add.at(dHe, graph.eb, dX[:, :H])
        np.add.at(dHe, graph.ea, dX[:, H:2 * H])
        dH = dH + dHe
    put("ein", xe, dE * (cache["E"][0] > 0))
    put("nin", xn, dH * (cache["H"][0] > 0))
    g = np.zeros(NWEIGHTS)
    for name, (o, k, n) in LAYOUT.items():
        g[o:o + (k + 1) * n] = grads[name].reshape(-1)
    return g


def loss_and_grad(w, graph, xe, xn, seed):
    coef, cache = forward(w, graph, xe, xn)
    loss, dcoef = probe_loss(graph, xe, coef, seed)
    return loss, backward(w, graph, xe, xn, cache, dcoef), coef


def gauge_basis(R, T):
    """Z (6N x 7): the camera parts of the world similarity motions (translation t, rotation w,
    scale s) under the update T += dT, R <- Rodrigues(w) R: dT_i = -R_i t + s T_i, w_i = -R_i w."""
    R = np.asarray(R).reshape(-1, 3, 3)
    T = np.asarray(T).reshape(-1, 3)
    N = R.shape[0]
    Z = np.zeros((6 * N, 7))
    for i in range(N):
        Z[6 * i:6 * i + 3, 0:3] = -R[i]
        Z[6 * i + 3:6 * i + 6, 3:6] = -R[i]
        Z[6 * i:6 * i + 3, 6] = T[i]
    return Z
