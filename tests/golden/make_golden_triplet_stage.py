"""Generates tests/golden/triplets/stage.npz: the reference's triplet stage
(SfM/generate_triples/src/generate_triples.cpp:380-415: triangulateLinear, the reprojection
filter, the survival tests, StdMetricBundleOptimizer for 5 iterations) on seeded triplets, run
through oracle/_ref/libv3dref.so (the reference compiled from its sources; the filter, which
lives in the application file, is restated there on the reference's own types).

    python tests/golden/make_golden_triplet_stage.py

Ragged arrays are stored concatenated with per-triplet offsets.  Cases: accepted triplets,
triplets with too few tracks, a triplet dominated by wrong matches (dropped by the ratio test),
an empty triplet, and tracks seen in two views only.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.bindings import Reference  # noqa: E402
from v3dsfmtoolkit_b200 import scenes  # noqa: E402


def cases():
    trips = scenes.triplet_stage_batch(n_triplets=20, seed=41, min_tracks=20, max_tracks=260)
    trips += scenes.triplet_stage_batch(n_triplets=2, seed=42, min_tracks=120, max_tracks=200, bad_frac=1.0)
    trips += scenes.triplet_stage_batch(n_triplets=2, seed=43, min_tracks=300, max_tracks=320, bad_frac=1.0,
                                        bad_outlier_frac=0.3)
    e = trips[0]
    trips.append(scenes.TripletTracks(e.R, e.T, e.focal, np.zeros(1, np.int32), np.zeros(0, np.int32),
                                      np.zeros((0, 2), np.float32)))
    return trips


def pack(trips):
    tp_off, m_off = [0], [0]
    for t in trips:
        tp_off.append(tp_off[-1] + t.n_tracks + 1)
        m_off.append(m_off[-1] + int(t.track_ptr[-1]))
    return dict(
        R=np.stack([t.R for t in trips]), T=np.stack([t.T for t in trips]), focal=np.stack([t.focal for t in trips]),
        track_ptr=np.concatenate([t.track_ptr for t in trips]), view=np.concatenate([t.view for t in trips]),
        pos=np.concatenate([t.pos for t in trips]).astype(np.float32), tp_off=np.array(tp_off), m_off=np.array(m_off))


def main():
    trips = cases()
    ref = Reference()
    outs = [ref.triplet_stage(t) for t in trips]
    d = pack(trips)
    d.update(verdict=np.array([o["verdict"] for o in outs]), n_points=np.array([o["n_points"] for o in outs]),
             status=np.array([o["status"] for o in outs]), iterations=np.array([o["iterations"] for o in outs]),
             cost=np.array([o["cost"] for o in outs]), R_out=np.stack([o["R"] for o in outs]),
             T_out=np.stack([o["T"] for o in outs]),
             X_out=np.concatenate([o["X"].reshape(-1, 3) for o in outs]),
             kept=np.concatenate([o["kept"] for o in outs]).astype(np.uint8))
    os.makedirs(os.path.join(HERE, "triplets"), exist_ok=True)
    np.savez_compressed(os.path.join(HERE, "triplets", "stage.npz"), **d)
    print("verdicts", np.bincount(d["verdict"], minlength=3), "tracks", int(d["tp_off"][-1] - len(trips)),
          "measurements", int(d["m_off"][-1]))


if __name__ == "__main__":
    main()
