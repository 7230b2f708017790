"""Training data, training and evaluation of the learned PCG preconditioner.

The network and every kernel it runs live in ``csrc/precond_gnn.cu`` (and the PCG solve in
``csrc/pcg.cu``) behind the C-ABI; this module only drives them:

  * :func:`training_scenes` -- seeded scenes of 100-2,000 cameras shaped like the two large
    workloads: forward-moving sequences with shared intrinsics (6-parameter cameras) and
    clustered groups with sparse inter-group co-visibility;
  * :func:`capture` -- runs the adjuster's own LM iterations (PCG, block-Jacobi) on a scene and
    captures its damped reduced camera systems over the range of damping the LM loop visits;
  * :func:`train` -- Adam over the captured set with the hand-written forward/backward kernels;
  * :func:`evaluate` -- PCG iterations with block-Jacobi, block-Jacobi + gauge space, the learned
    factor, and the learned factor + gauge space.

Command line (on a GPU):

  python -m v3dsfmtoolkit_b200.precond train --systems 500 --epochs 30 --out <weights.npy>
  python -m v3dsfmtoolkit_b200.precond evaluate --weights <weights.npy>
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import capi, scenes

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "precond_weights.npy")
VARIANTS = ("jacobi", "jacobi_gauge", "learned", "learned_gauge")


def training_scenes(seed, n_min=100, n_max=2000, points_per_cam=100):
    """One seeded scene: even seeds give a sequence, odd seeds a clustered scene."""
    rng = np.random.default_rng(seed)
    N = int(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
    if seed % 2 == 0:
        return scenes.sequence_scene(n_cams=N, n_points=points_per_cam * N, mode=scenes.FULL_BUNDLE_METRIC,
                                     seed=seed, outlier_frac=0.0)
    per = int(rng.integers(20, 101))
    groups = max(1, N // per)
    return scenes.cluster_scene(n_groups=groups, cams_per_group=per, n_points=points_per_cam * groups * per,
                                seed=seed)


def capture(pset, sc, n_captures, iterations=20, span=(0.0, 4.0), max_pcg=500):
    """Adds up to `n_captures` systems of `sc` to `pset`: the adjuster runs `iterations` LM
    iterations (PCG, block-Jacobi, mixed precision) and its reduced system at the reached
    parameters is captured at dampings lambda_end * 10^u, u evenly spread over `span` -- from the
    final damping up to the early iterations' range, which is where the solver spends its PCG
    iterations.  A damping at which a diagonal camera block is not numerically positive
    definite is skipped.  Returns the number of systems added."""
    h = capi.Handle.from_scene(sc)
    added = 0
    try:
        r = h.minimize(max_iterations=iterations, solver=capi.SOLVER_PCG, pcg_max_iterations=max_pcg)
        for u in np.linspace(span[0], span[1], n_captures):
            try:
                pset.capture(h, r.lambda_ * 10.0 ** u)
                added += 1
            except capi.V3dbaError as e:
                if e.code != capi.ERR_INVALID_INPUT:
                    raise
        return added
    finally:
        h.close()


def train(pset, epochs=30, lr=1e-3, seed=0, model=None):
    model = capi.PrecondModel(seed=seed) if model is None else model
    hist = model.train(pset, epochs, lr, seed)
    return model, hist


def evaluate(pset, model, tol=1e-6, max_iter=5000, rhs_seed=0):
    """PCG iteration counts of every system in `pset`: an (n, 4) array over VARIANTS; -1 where
    a variant does not apply.  rhs_seed 0 solves with each captured system's own right-hand side
    (the LM's reduced gradient, which has no component along the gauge motions); a positive seed
    uses seeded random right-hand sides instead (seed + index)."""
    out = []
    for i in range(len(pset)):
        d = pset.pcg_iterations(i, model, tol=tol, max_iter=max_iter, rhs_seed=rhs_seed + i if rhs_seed else 0)
        out.append([(-1 if d[k] is None else d[k]) for k in VARIANTS])
    return np.array(out, dtype=np.int64).reshape(-1, 4)


def summarize(ev):
    """Total iterations per variant and the cuts against block-Jacobi."""
    tot = {k: int(ev[:, j].sum()) for j, k in enumerate(VARIANTS) if np.all(ev[:, j] >= 0)}
    cut = {f"cut_{k}_vs_jacobi": round(tot["jacobi"] / max(v, 1), 3) for k, v in tot.items() if k != "jacobi"}
    return {**{f"{k}_iterations": v for k, v in tot.items()}, **cut}


def _main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("--systems", type=int, default=500)
    ap.add_argument("--per-scene", type=int, default=10)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed-base", type=int, default=1000)
    ap.add_argument("--eval-seed-base", type=int, default=900000)
    ap.add_argument("--eval-scenes", type=int, default=6)
    ap.add_argument("--n-max", type=int, default=2000)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--weights", default=WEIGHTS)
    ap.add_argument("--report", default=None)
    a = ap.parse_args()
    import torch
    torch.cuda.set_device(0)
    t0 = time.time()
    report = {}
    if a.cmd == "train":
        pset = capi.PrecondSet()
        s = a.seed_base
        while len(pset) < a.systems:
            capture(pset, training_scenes(s, n_max=a.n_max), min(a.per_scene, a.systems - len(pset)))
            s += 1
        report["train_systems"] = len(pset)
        report["train_scenes"] = s - a.seed_base
        report["capture_s"] = round(time.time() - t0, 1)
        print(f"captured {len(pset)} systems from {s - a.seed_base} scenes in {time.time() - t0:.0f}s", flush=True)
        t1 = time.time()
        model, hist = train(pset, a.epochs, a.lr, seed=0)
        report["train_s"] = round(time.time() - t1, 1)
        report["loss_per_epoch"] = [round(float(x), 6) for x in hist]
        print("loss per epoch", np.round(hist, 5).tolist(), flush=True)
        np.save(a.out, model.weights())
        a.weights = a.out
    model = capi.PrecondModel.load(a.weights)
    untrained = capi.PrecondModel(seed=0)
    eset = capi.PrecondSet()
    for s in range(a.eval_seed_base, a.eval_seed_base + a.eval_scenes):
        capture(eset, training_scenes(s, n_max=a.n_max), 4)
    report["eval_systems"] = len(eset)
    report["lm_rhs"] = {"trained": summarize(evaluate(eset, model)), "untrained": summarize(evaluate(eset, untrained))}
    report["random_rhs"] = {"trained": summarize(evaluate(eset, model, rhs_seed=1)),
                            "untrained": summarize(evaluate(eset, untrained, rhs_seed=1))}
    print(json.dumps(report), flush=True)
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    _main()
