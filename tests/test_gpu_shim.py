"""The drop-in C++ header (include/v3d_b200/v3d_metricbundle.h) used the way the reference's
pipeline uses its optimizer: tests/shim/shim_demo.cpp is compiled against the reference's own
headers, constructs the optimizer classes with the reference's signatures and calls minimize().
Its results must match the reference's (golden fixtures)."""
import os
import struct
import subprocess
import tempfile

import numpy as np
import pytest

from v3dsfmtoolkit_b200 import capi
from tests.helpers import golden_names, load_golden, load_rotation_golden, param_rel, rotation_golden_names

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEMO = os.path.join(ROOT, "tests", "shim", "_build", "shim_demo")
ROT_DEMO = os.path.join(ROOT, "tests", "shim", "_build", "rotations_demo")
STEREO_DEMO = os.path.join(ROOT, "tests", "shim", "_build", "stereo_demo")


def _write_scene(path, sc, max_iterations, precision, nv):
    with open(path, "wb") as f:
        f.write(struct.pack("<10i", sc.model, sc.mode, sc.n_cams, sc.n_points, sc.n_obs, max_iterations,
                            precision, *nv))
        f.write(struct.pack("<d", sc.inlier_threshold))
        for a in (sc.K, sc.R, sc.T):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        if sc.dist is not None:
            f.write(np.ascontiguousarray(sc.dist, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(sc.X, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(sc.meas, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(sc.view, dtype=np.int32).tobytes())
        f.write(np.ascontiguousarray(sc.point, dtype=np.int32).tobytes())


def _read_out(path, sc):
    b = open(path, "rb").read()
    status, iters = struct.unpack_from("<2i", b, 0)
    off = 8
    out = []
    for shape in (sc.K.shape, sc.R.shape, sc.T.shape, None if sc.dist is None else sc.dist.shape, sc.X.shape):
        if shape is None:
            out.append(None)
            continue
        n = int(np.prod(shape))
        out.append(np.frombuffer(b, dtype=np.float64, count=n, offset=off).reshape(shape))
        off += 8 * n
    return status, iters, out


@pytest.mark.skipif(not os.path.exists(DEMO), reason="shim demo not built (needs the reference headers at build time)")
@pytest.mark.parametrize("name", [n for n in golden_names() if not n.startswith("stereo")])
def test_dropin_header_matches_reference(name):
    sc, g = load_golden(name)
    nv = tuple(int(v) for v in g["nonvarying"])
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "scene.bin"), os.path.join(d, "out.bin")
        _write_scene(sp, sc, int(g["max_iterations"]), capi.PRECISION_FP64, nv)
        r = subprocess.run([DEMO, sp, op], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        status, iters, (K, R, T, dist, X) = _read_out(op, sc)
    assert status == int(g["status"])
    assert iters == int(g["iterations"])
    assert param_rel((K, R, T, X), (g["K"], g["R"], g["T"], g["X"])) < 1e-5
    if sc.dist is not None:
        assert param_rel((dist,), (g["dist"],)) < 1e-4 or np.abs(dist - g["dist"]).max() < 1e-9


@pytest.mark.skipif(not os.path.exists(ROT_DEMO), reason="rotation demo not built (needs the reference headers at build time)")
@pytest.mark.parametrize("name", rotation_golden_names())
def test_rotation_header_matches_reference(name):
    """V3D::B200::refineConsistentRotations called on the reference's own container types gives
    the reference's refined rotations (golden fixtures)."""
    graph, g = load_rotation_golden(name)
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "graph.bin"), os.path.join(d, "out.bin")
        with open(sp, "wb") as f:
            f.write(struct.pack("<2i", graph.n_views, graph.n_pairs))
            f.write(np.ascontiguousarray(graph.rel, dtype=np.float64).tobytes())
            f.write(np.ascontiguousarray(graph.pairs, dtype=np.int32).tobytes())
            f.write(np.ascontiguousarray(graph.R0, dtype=np.float64).tobytes())
        r = subprocess.run([ROT_DEMO, sp, op], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        b = open(op, "rb").read()
    assert struct.unpack_from("<i", b, 0)[0] == capi.OK
    R = np.frombuffer(b, dtype=np.float64, offset=4).reshape(-1, 3, 3)
    assert np.abs(R - g["R"]).max() < 1e-5


@pytest.mark.skipif(not os.path.exists(STEREO_DEMO), reason="stereo demo not built (needs the reference headers at build time)")
@pytest.mark.parametrize("name", [n for n in golden_names() if n.startswith("stereo")])
def test_stereo_header_matches_reference(name):
    """include/v3d_b200/v3d_stereobundle.h driven the way the reference's rig adjuster is
    constructed and minimised gives the reference's status, iterations and parameters."""
    sc, g = load_golden(name)
    nv = tuple(int(v) for v in g["nonvarying"])
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "scene.bin"), os.path.join(d, "out.bin")
        with open(sp, "wb") as f:
            f.write(struct.pack("<8i", sc.n_cams, sc.n_points, sc.n_obs, sc.n_rig, int(g["max_iterations"]),
                                capi.PRECISION_FP64, nv[0], nv[1]))
            f.write(struct.pack("<d", sc.inlier_threshold))
            for a in (sc.R, sc.T, sc.X, sc.meas, sc.rig_K, sc.rig_R, sc.rig_T):
                f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
            for a in (sc.view, sc.point, sc.sub):
                f.write(np.ascontiguousarray(a, dtype=np.int32).tobytes())
        r = subprocess.run([STEREO_DEMO, sp, op], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        b = open(op, "rb").read()
    status, iters = struct.unpack_from("<2i", b, 0)
    N, M = sc.n_cams, sc.n_points
    vals = np.frombuffer(b, dtype=np.float64, offset=8)
    R, T, X = vals[:9 * N].reshape(N, 3, 3), vals[9 * N:12 * N].reshape(N, 3), vals[12 * N:].reshape(M, 3)
    assert status == int(g["status"]) and iters == int(g["iterations"])
    assert param_rel((R, T, X), (g["R"], g["T"], g["X"])) < 1e-5



POINTS_DEMO = os.path.join(ROOT, "tests", "shim", "_build", "points_demo")


@pytest.mark.skipif(not os.path.exists(POINTS_DEMO), reason="points demo not built (needs the reference headers)")
@pytest.mark.parametrize("seed", [1, 2])
def test_dropin_bundle_point_structure_matches_reference_struct(seed):
    """include/v3d_b200/v3d_bundlepoints.h against the reference's inline BundlePointStructure in
    one C++ caller: identical members after the constructor (thresholds -1 .. 5, empty and long
    tracks) and identical reconstructions after createPointStructure in both branches."""
    r = subprocess.run([POINTS_DEMO, str(seed)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout
