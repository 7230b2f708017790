"""Runs the reference optimizer (compiled from its sources, oracle/_ref) on the bench workloads
and records its final cost, status and iteration count in tests/golden/bench_reference.json.

    python tests/golden/make_bench_reference.py

The bench's time-to-reference-cost target is this cost times (1 + 1e-6).  The scenes are
regenerated from their seeds by v3dsfmtoolkit_b200.scenes; the json also stores a checksum of
the generated inputs so that a changed generator is detected.
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.bindings import Reference  # noqa: E402
from v3dsfmtoolkit_b200 import scenes  # noqa: E402

WORKLOADS = {
    "circle20": (lambda: scenes.circle_scene(), 100),
    "sequence200": (lambda: scenes.sequence_scene(), 100),
    "stereo300": (lambda: scenes.stereo_rig_scene(n_poses=300, n_points=40000, seed=0, window=6, outlier_frac=0.01), 40),
}


def scene_digest(sc):
    h = hashlib.sha256()
    for a in (sc.K, sc.R, sc.T, sc.X, sc.meas, sc.view, sc.point):
        h.update(np.ascontiguousarray(a).tobytes())
    if sc.dist is not None:
        h.update(np.ascontiguousarray(sc.dist).tobytes())
    if getattr(sc, "rig_K", None) is not None:
        for a in (sc.rig_K, sc.rig_R, sc.rig_T, sc.sub):
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def main(names):
    ref = Reference()
    path = os.path.join(HERE, "bench_reference.json")
    out = json.load(open(path)) if os.path.exists(path) else {}
    for name in names:
        make, iters = WORKLOADS[name]
        sc = make()
        t0 = time.perf_counter()
        params, info = ref.minimize(sc, max_iterations=iters)
        dt = time.perf_counter() - t0
        cost = ref.cost(sc, params)
        out[name] = dict(cost=cost, status=info["status"], iterations=info["iterations"],
                         n_rejected=info["n_rejected"], n_relinearizations=info["n_relinearizations"],
                         max_iterations=iters, wall_s_1core=dt, digest=scene_digest(sc),
                         n_cams=sc.n_cams, n_points=sc.n_points, n_obs=sc.n_obs,
                         trace_cost=[float(c) for c in info["trace_cost"]])
        print(name, out[name]["cost"], out[name]["status"], out[name]["iterations"], f"{dt:.1f}s")
    json.dump(out, open(path, "w"), indent=1)


if __name__ == "__main__":
    main(sys.argv[1:] or list(WORKLOADS))
