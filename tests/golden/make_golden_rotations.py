"""Generates the rotation-averaging fixtures of tests/golden/rotations/ by running the
reference's own V3D::refineConsistentRotations (SparseRotationOptimizer, compiled from its
sources into oracle/_ref/libv3dref.so, see oracle/Makefile) on small seeded view graphs.

    python tests/golden/make_golden_rotations.py

Each fixture stores the graph (relative rotations, view pairs, initial rotations), the
reference's refined rotations and its cost trace (the |residual|^2 line minimize() prints once
per relinearization).  The status and iteration count are not visible through the reference's
function; the fixture stores those of the C restatement (oracle/v3dba_oracle.c), which must
reproduce the reference's rotations and trace bit for bit on every case.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.bindings import Reference, Restatement  # noqa: E402
from v3dsfmtoolkit_b200 import scenes  # noqa: E402

OUT = os.path.join(HERE, "rotations")


def edge_graph():
    """Isolated view, duplicated pair, a self-pair and both pair orientations."""
    g = scenes.rotation_graph(n_views=10, n_pairs=18, seed=21, init_deg=8.0)
    pairs = g.pairs.copy()
    pairs[pairs == 9] = 8                      # view 9 keeps no pair
    extra = np.array([pairs[0], pairs[0][::-1], [3, 3]], dtype=np.int32)
    pairs = np.concatenate([pairs, extra])
    rel = g.R_true[pairs[:, 1]] @ np.transpose(g.R_true[pairs[:, 0]], (0, 2, 1))
    rel = scenes.rodrigues(np.random.default_rng(5).normal(scale=0.01, size=(len(pairs), 3))) @ rel
    return scenes.RotationGraph(rel, pairs, g.R0, g.R_true, name="rot_edges")


def exact_graph():
    """Noise-free graph started at the true rotations: converged at the first gradient test."""
    g = scenes.rotation_graph(n_views=15, n_pairs=40, seed=22, noise_deg=0.0, init_deg=0.0)
    return scenes.RotationGraph(g.rel, g.pairs, g.R_true.copy(), g.R_true, name="rot_exact")


CASES = {
    "rot_small": lambda: scenes.rotation_graph(n_views=12, n_pairs=20, seed=2, init_deg=20.0),
    "rot_graph": lambda: scenes.rotation_graph(n_views=30, n_pairs=120, seed=1),
    "rot_outliers": lambda: scenes.rotation_graph(n_views=50, n_pairs=400, seed=3, outlier_frac=0.1),
    "rot_medium": lambda: scenes.rotation_graph(n_views=200, n_pairs=2000, seed=4),
    "rot_chain": lambda: scenes.rotation_graph(n_views=60, n_pairs=60, window=1, seed=6, init_deg=25.0),
    "rot_edges": edge_graph,
    "rot_exact": exact_graph,
}


def main():
    os.makedirs(OUT, exist_ok=True)
    ref, orc = Reference(), Restatement()
    for name, make in CASES.items():
        g = make()
        R, trace = ref.refine_rotations(g)
        Ro, info = orc.rotations_minimize(g)
        same = np.array_equal(R, Ro) and np.array_equal(trace, info["trace_cost"])
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), rel=g.rel, pairs=g.pairs, R0=g.R0, R=R, trace=trace,
                            status=info["status"], iterations=info["iterations"], n_rejected=info["n_rejected"])
        print(f"{name}: views={g.n_views} pairs={g.n_pairs} relin={len(trace)} status={info['status']} "
              f"it={info['iterations']} cost={trace[-1] if len(trace) else float('nan'):.12g} restatement_exact={same}")


if __name__ == "__main__":
    main()
