"""Generates the golden fixtures of tests/golden/ by running the reference optimizer compiled from
its own sources (oracle/_ref/libv3dref.so, see oracle/Makefile) on small seeded scenes.

    python tests/golden/make_golden.py

Each fixture stores the scene inputs and the reference's outputs: per-observation residuals,
weights and Jacobians at the initial parameters, and the result of minimize() (final parameters,
status, iteration count, per-relinearisation cost/lambda trace).  The reference ships no test
vectors of its own, so these are the pinned known answers for the oracle and the GPU path.

Every case runs in a fresh process: with fixed cameras and points the reference accumulates
Jacobian blocks it never filled (uninitialised heap memory) into W_0
(V3D/src/Math/v3d_optimization.cpp:313, 930), so its result for std_fixed depends on what the
heap held before; a fresh process gives the zero-filled (clean) run.
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.bindings import Reference  # noqa: E402
from v3dsfmtoolkit_b200 import scenes  # noqa: E402

CASES = {
    # name: (scene factory, max_iterations, nonvarying)
    "std_circle": (lambda: scenes.circle_scene(n_cams=8, n_points=240, seed=11), 50, (0, 0, 0)),
    "std_circle_huber": (lambda: scenes.circle_scene(n_cams=6, n_points=150, seed=12, inlier_threshold=1.0), 30, (0, 0, 0)),
    "std_fixed": (lambda: scenes.circle_scene(n_cams=6, n_points=150, seed=13), 30, (1, 5, 0)),
    "common_rt": (lambda: scenes.sequence_scene(n_cams=8, n_points=300, seed=14), 25, (0, 0, 0)),
    "common_radial": (lambda: scenes.sequence_scene(n_cams=8, n_points=300, seed=15, mode=3), 25, (0, 0, 0)),
    "common_focal": (lambda: scenes.sequence_scene(n_cams=8, n_points=300, seed=16, mode=1), 25, (0, 0, 1)),
    "common_norot": (lambda: scenes.sequence_scene(n_cams=8, n_points=300, seed=17, mode=-1), 25, (0, 0, 0)),
    "varying_rt": (lambda: scenes.varying_scene(n_cams=6, n_points=200, seed=18, mode=4), 25, (0, 0, 0)),
    "varying_pp": (lambda: scenes.varying_scene(n_cams=6, n_points=200, seed=19, mode=2), 25, (0, 0, 0)),
    "stereo_rig": (lambda: scenes.stereo_rig_scene(n_poses=10, n_points=300, seed=20), 30, (0, 0, 0)),
    "stereo_huber": (lambda: scenes.stereo_rig_scene(n_poses=8, n_points=250, seed=24, outlier_frac=0.03,
                                                     inlier_threshold=2.0), 40, (0, 0, 0)),
    "stereo_fixed": (lambda: scenes.stereo_rig_scene(n_poses=8, n_points=250, seed=22), 60, (1, 4, 0)),
}


NLIN = 256   # per-observation linearisation stored for the first NLIN observations


def main():
    if len(sys.argv) > 2 and sys.argv[1] == "--case":
        return make_case(sys.argv[2])
    for name in CASES:
        subprocess.run([sys.executable, os.path.abspath(__file__), "--case", name], check=True)


def make_case(name):
    ref = Reference()
    for name, (make, iters, nv) in [(name, CASES[name])]:
        sc = make()
        e, w, A, B, Cm = ref.linearize(sc)
        (K, R, T, dist, X), info = ref.minimize(sc, max_iterations=iters, nonvarying=nv)
        cost = ref.cost(sc, (K, R, T, dist, X))
        rig = {}
        if sc.model == scenes.MODEL_STEREO:
            rig = dict(rig_K=sc.rig_K, rig_R=sc.rig_R, rig_T=sc.rig_T, sub=sc.sub)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"), **rig,
            model=sc.model, mode=sc.mode, inlier_threshold=sc.inlier_threshold,
            K0=sc.K, R0=sc.R, T0=sc.T, dist0=sc.dist if sc.dist is not None else np.zeros(0), X0=sc.X,
            meas=sc.meas, view=sc.view, point=sc.point, max_iterations=iters, nonvarying=np.array(nv),
            e=e[:NLIN], w=w[:NLIN], A=A[:NLIN], B=B[:NLIN], C=Cm[:NLIN],
            K=K, R=R, T=T, dist=dist, X=X, cost=cost, status=info["status"], iterations=info["iterations"],
            n_rejected=info["n_rejected"], trace_cost=info["trace_cost"], trace_lambda=info["trace_lambda"])
        print(f"{name}: N={sc.n_cams} M={sc.n_points} K={sc.n_obs} status={info['status']} "
              f"it={info['iterations']} cost={cost:.12g}")


if __name__ == "__main__":
    main()
