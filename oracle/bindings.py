"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the CPU oracle.

* :class:`Reference` -- the reference's own optimizer compiled from its sources
  (``oracle/_ref/libv3dref.so``, built by ``oracle/Makefile`` where the reference is mounted;
  the prebuilt file travels with the repository snapshot).
* :class:`Restatement` -- the plain-C FP64 restatement (``oracle/_build/libv3dba_oracle.so``).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this
module, and only as the checker / the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libv3dref.so")
ORC_LIB = os.path.join(HERE, "_build", "libv3dba_oracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _scene_arrays(scene):
    K, R, T, dist, X = (np.array(a, dtype=np.float64, copy=True) for a in scene.params())
    return K, R, T, dist, X


def build(quiet=True):
    """Builds whatever oracle/Makefile can build here (the reference part needs its sources)."""
    import subprocess
    cmd = ["make", "-C", HERE]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)


def reference_available() -> bool:
    return os.path.exists(REF_LIB)


class Reference:
    """The reference optimizer classes driven through oracle/ref_capi.cpp."""

    def __init__(self, path=REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference oracle library missing: {path} (run make -C oracle)")
        self.lib = C.CDLL(path)
        L = self.lib
        L.v3dref_minimize.restype = C.c_int
        L.v3dref_minimize.argtypes = [C.c_int] * 5 + [C.c_double] + [_dp] * 5 + [_dp, _ip, _ip] + \
            [C.c_int] * 3 + [C.c_double, C.c_int, C.c_int] + [_ip, _ip, _dp] + [_dp, _dp, _ip, C.c_int, _ip, _ip]
        L.v3dref_linearize.restype = C.c_int
        L.v3dref_linearize.argtypes = [C.c_int] * 5 + [C.c_double] + [_dp] * 5 + [_dp, _ip, _ip] + [_dp] * 5
        L.v3dref_cost.restype = C.c_double
        L.v3dref_cost.argtypes = [C.c_int] * 5 + [C.c_double] + [_dp] * 5 + [_dp, _ip, _ip]
        L.v3dref_minimize_stereo.restype = C.c_int
        L.v3dref_minimize_stereo.argtypes = [C.c_int] * 4 + [C.c_double] + [_dp] * 4 + [_ip] * 3 + [_dp] * 3 + \
            [C.c_int, C.c_int, C.c_double, C.c_int, _ip, _ip, _dp, _dp, _dp, _ip, C.c_int, _ip, _ip]
        L.v3dref_linearize_stereo.restype = C.c_int
        L.v3dref_linearize_stereo.argtypes = [C.c_int] * 4 + [C.c_double] + [_dp] * 4 + [_ip] * 3 + [_dp] * 7
        L.v3dref_triplet_stage.restype = C.c_int
        L.v3dref_triplet_stage.argtypes = [_dp, _dp, _dp, C.c_int, _ip, _ip, C.POINTER(C.c_float), C.c_double,
                                           C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                           _ip, _ip, _ip, _ip, _dp, _dp, _dp, _dp, C.POINTER(C.c_ubyte)]
        L.v3dref_refine_rotations.restype = C.c_int
        L.v3dref_refine_rotations.argtypes = [C.c_int, C.c_int, _dp, _ip, _dp, _dp, C.c_int, _ip]

    def _head(self, sc):
        return (sc.model, sc.mode, sc.n_cams, sc.n_points, sc.n_obs, float(sc.inlier_threshold))

    def _stereo_args(self, sc):
        return (_f64(sc.meas), _i32(sc.view), _i32(sc.point), _i32(sc.sub), _f64(sc.rig_K), _f64(sc.rig_R),
                _f64(sc.rig_T))

    def _minimize_stereo(self, scene, tau, max_iterations, nonvarying, trace_cap):
        K, R, T, dist, X = _scene_arrays(scene)
        m, v, p, s, rk, rr, rt = self._stereo_args(scene)
        st, it, lam = C.c_int(), C.c_int(), C.c_double()
        tc, tl, ti = np.zeros(trace_cap), np.zeros(trace_cap), np.zeros(trace_cap, dtype=np.int32)
        tlen, nrej = C.c_int(), C.c_int()
        self.lib.v3dref_minimize_stereo(scene.n_cams, scene.n_points, scene.n_obs, scene.n_rig,
                                        float(scene.inlier_threshold), _d(R), _d(T), _d(X), _d(m), _i(v), _i(p),
                                        _i(s), _d(rk), _d(rr), _d(rt), nonvarying[0], nonvarying[1], tau,
                                        max_iterations, C.byref(st), C.byref(it), C.byref(lam), _d(tc), _d(tl),
                                        _i(ti), trace_cap, C.byref(tlen), C.byref(nrej))
        n = min(tlen.value, trace_cap)
        info = dict(status=st.value, iterations=it.value, lambda_=lam.value,
                    trace_cost=tc[:n].copy(), trace_lambda=tl[:n].copy(), trace_iter=ti[:n].copy(),
                    n_relinearizations=tlen.value, n_rejected=nrej.value)
        return (K, R, T, dist, X), info

    def minimize(self, scene, tau=1e-3, max_iterations=50, nonvarying=(0, 0, 0), verbosity=0,
                 trace_cap=256):
        """Runs minimize() on a copy of ``scene``'s parameters; returns (params, info)."""
        if scene.model == 3:
            return self._minimize_stereo(scene, tau, max_iterations, nonvarying, trace_cap)
        K, R, T, dist, X = _scene_arrays(scene)
        meas, view, point = _f64(scene.meas), _i32(scene.view), _i32(scene.point)
        st, it, lam = C.c_int(), C.c_int(), C.c_double()
        tc, tl, ti = np.zeros(trace_cap), np.zeros(trace_cap), np.zeros(trace_cap, dtype=np.int32)
        tlen, nrej = C.c_int(), C.c_int()
        rc = self.lib.v3dref_minimize(*self._head(scene), _d(K), _d(R), _d(T), _d(dist), _d(X),
                                      _d(meas), _i(view), _i(point), *nonvarying, tau, max_iterations,
                                      verbosity, C.byref(st), C.byref(it), C.byref(lam),
                                      _d(tc), _d(tl), _i(ti), trace_cap, C.byref(tlen), C.byref(nrej))
        if rc != 0:
            raise ValueError("reference rejected the problem")
        n = min(tlen.value, trace_cap)
        info = dict(status=st.value, iterations=it.value, lambda_=lam.value,
                    trace_cost=tc[:n].copy(), trace_lambda=tl[:n].copy(), trace_iter=ti[:n].copy(),
                    n_relinearizations=tlen.value, n_rejected=nrej.value)
        return (K, R, T, dist, X), info

    def linearize(self, scene, params=None):
        dA, dC = scene.dims
        K, R, T, dist, X = params if params is not None else _scene_arrays(scene)
        n = scene.n_obs
        if scene.model == 3:
            m, v, p, s, rk, rr, rt = self._stereo_args(scene)
            e, w, A, B = np.zeros((n, 2)), np.zeros(n), np.zeros((n, 2, 6)), np.zeros((n, 2, 3))
            self.lib.v3dref_linearize_stereo(scene.n_cams, scene.n_points, n, scene.n_rig, float(scene.inlier_threshold),
                                             _d(_f64(R)), _d(_f64(T)), _d(_f64(X)), _d(m), _i(v), _i(p), _i(s),
                                             _d(rk), _d(rr), _d(rt), _d(e), _d(w), _d(A), _d(B))
            return e, w, A, B, np.zeros((n, 2, 0))
        e, w = np.zeros((n, 2)), np.zeros(n)
        A, B, Cm = np.zeros((n, 2, dA)), np.zeros((n, 2, 3)), np.zeros((n, 2, max(dC, 1)))
        rc = self.lib.v3dref_linearize(*self._head(scene), _d(_f64(K)), _d(_f64(R)), _d(_f64(T)),
                                       _d(_f64(dist)), _d(_f64(X)), _d(_f64(scene.meas)),
                                       _i(_i32(scene.view)), _i(_i32(scene.point)),
                                       _d(e), _d(w), _d(A), _d(B), _d(Cm) if dC else None)
        if rc != 0:
            raise ValueError("reference rejected the problem")
        return e, w, A, B, Cm[..., :dC]

    def cost(self, scene, params=None):
        K, R, T, dist, X = params if params is not None else _scene_arrays(scene)
        if scene.model == 3:
            e, w, _, _, _ = self.linearize(scene, (K, R, T, dist, X))
            return float(np.sum(w * w * np.sum(e * e, axis=1)))
        return self.lib.v3dref_cost(*self._head(scene), _d(_f64(K)), _d(_f64(R)), _d(_f64(T)),
                                    _d(_f64(dist)), _d(_f64(X)), _d(_f64(scene.meas)),
                                    _i(_i32(scene.view)), _i(_i32(scene.point)))


    def triplet_stage(self, trip, max_reproj_error=1.0, min_points=50, min_point_ratio=0.5, inlier_threshold=1.0,
                      tau=1e-3, max_iterations=5):
        """The reference's triplet stage (generate_triples.cpp:380-415) on one TripletTracks."""
        n = trip.n_tracks
        nm = int(trip.track_ptr[-1])
        v, ns, st, it = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        cost = C.c_double()
        Ro, To, X = np.zeros(27), np.zeros(9), np.zeros(3 * max(n, 1))
        kept = np.zeros(max(nm, 1), dtype=np.uint8)
        pos = np.ascontiguousarray(trip.pos, dtype=np.float32)
        self.lib.v3dref_triplet_stage(_d(_f64(trip.R)), _d(_f64(trip.T)), _d(_f64(trip.focal)), n,
                                      _i(_i32(trip.track_ptr)), _i(_i32(trip.view)),
                                      pos.ctypes.data_as(C.POINTER(C.c_float)), max_reproj_error, min_points,
                                      min_point_ratio, inlier_threshold, tau, max_iterations, C.byref(v),
                                      C.byref(ns), C.byref(st), C.byref(it), C.byref(cost), _d(Ro), _d(To),
                                      _d(X), kept.ctypes.data_as(C.POINTER(C.c_ubyte)))
        return dict(verdict=v.value, n_points=ns.value, status=st.value, iterations=it.value, cost=cost.value,
                    R=Ro.reshape(3, 3, 3), T=To.reshape(3, 3), X=X[:3 * n].reshape(n, 3), kept=kept[:nm].copy())

    def bundle_point_structure(self, tracks, n_required=2):
        """The reference's BundlePointStructure(reconstruction, nRequiredMeasurements) on tracks
        (dict: track_ptr, pos (n, 3), view, id, mpos (K, 2) float32); returns its flat arrays."""
        return _bps_call(self.lib.v3dref_bundle_point_structure, tracks, n_required)

    def create_point_structure(self, bps, from_scratch, tracks=None):
        """The reference's BundlePointStructure::createPointStructure; returns the tracks."""
        return _cps_call(self.lib.v3dref_create_point_structure, bps, from_scratch, tracks)

    def refine_rotations(self, graph, rotations=None, trace_cap=512):
        """V3D::refineConsistentRotations on a copy of the graph's initial rotations; returns
        (rotations (n, 3, 3), err per relinearization as printed by the reference)."""
        R = np.array(graph.R0 if rotations is None else rotations, dtype=np.float64, copy=True)
        tr, tlen = np.zeros(trace_cap), C.c_int()
        self.lib.v3dref_refine_rotations(graph.n_views, graph.n_pairs, _d(_f64(graph.rel)), _i(_i32(graph.pairs)),
                                         _d(R), _d(tr), trace_cap, C.byref(tlen))
        return R, tr[:min(tlen.value, trace_cap)].copy()


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None


def _bps_call(fn, tracks, n_required):
    """Calls a BundlePointStructure producer with the C signature of v3dba_bundle_point_structure
    (the reference wrapper and the GPU entry point share it)."""
    ptr = _i32(tracks["track_ptr"])
    n = ptr.size - 1
    K = int(ptr[-1])
    pos, view, ids = _f64(tracks["pos"]), _i32(tracks["view"]), _i32(tracks["id"])
    mpos = np.ascontiguousarray(tracks["mpos"], dtype=np.float32)
    npts, nm = C.c_int(), C.c_int()
    pts, meas = np.zeros((max(n, 1), 3)), np.zeros((max(K, 1), 2))
    mid, cv, cp, xs = (np.zeros(max(K, 1), np.int32), np.zeros(max(K, 1), np.int32), np.zeros(max(K, 1), np.int32),
                       np.zeros(max(n, 1), np.int32))
    rc = fn(n, _i(ptr), _d(pos), _i(view), _i(ids), _fp(mpos), int(n_required), C.byref(npts), C.byref(nm), _d(pts),
            _d(meas), _i(mid), _i(cv), _i(cp), _i(xs))
    if rc != 0:
        raise ValueError(f"BundlePointStructure failed: {rc}")
    M, Kk = npts.value, nm.value
    return dict(points3d=pts[:M].copy(), measurements=meas[:Kk].copy(), measurement_ids=mid[:Kk].copy(),
                corresponding_view=cv[:Kk].copy(), corresponding_point=cp[:Kk].copy(), xs_indices=xs[:M].copy())


def _cps_call(fn, bps, from_scratch, tracks):
    """Calls a createPointStructure with the C signature of v3dba_create_point_structure."""
    pts, meas = _f64(bps["points3d"]).reshape(-1, 3), _f64(bps["measurements"]).reshape(-1, 2)
    M, K = pts.shape[0], meas.shape[0]
    mid, cv, cp = _i32(bps["measurement_ids"]), _i32(bps["corresponding_view"]), _i32(bps["corresponding_point"])
    xs = _i32(bps["xs_indices"])
    if from_scratch:
        ptr, pos = np.zeros(M + 1, np.int32), np.zeros((max(M, 1), 3))
        view, ids, mpos = np.zeros(max(K, 1), np.int32), np.zeros(max(K, 1), np.int32), np.zeros((max(K, 1), 2), np.float32)
        n = M
    else:
        ptr = _i32(tracks["track_ptr"]).copy()
        n = ptr.size - 1
        pos = _f64(tracks["pos"]).copy()
        view, ids = _i32(tracks["view"]).copy(), _i32(tracks["id"]).copy()
        mpos = np.ascontiguousarray(tracks["mpos"], dtype=np.float32).copy()
    rc = fn(1 if from_scratch else 0, M, K, _d(pts), _d(meas), _i(mid), _i(cv), _i(cp), _i(xs), n, _i(ptr), _d(pos),
            _i(view), _i(ids), _fp(mpos))
    if rc != 0:
        raise ValueError(f"createPointStructure failed: {rc}")
    Kt = int(ptr[-1])
    return dict(track_ptr=ptr, pos=pos[:n].copy(), view=view[:Kt].copy(), id=ids[:Kt].copy(), mpos=mpos[:Kt].copy())


class _OrcProblem(C.Structure):
    _fields_ = [("model", C.c_int), ("mode", C.c_int), ("n_cams", C.c_int), ("n_points", C.c_int),
                ("n_obs", C.c_int), ("inlier_threshold", C.c_double), ("nnA", C.c_int),
                ("nnB", C.c_int), ("nnC", C.c_int), ("meas", _dp), ("view", _ip), ("point", _ip),
                ("n_rig", C.c_int), ("rig_K", _dp), ("rig_R", _dp), ("rig_T", _dp), ("sub", _ip)]


class _OrcParams(C.Structure):
    _fields_ = [("K", _dp), ("R", _dp), ("T", _dp), ("dist", _dp), ("X", _dp)]


class _OrcOptions(C.Structure):
    _fields_ = [("tau", C.c_double), ("max_iterations", C.c_int), ("gradient_threshold", C.c_double),
                ("update_threshold", C.c_double), ("param_length", C.c_double),
                ("cached_aspect_ratio", C.c_double), ("lambda_", C.c_double), ("nu", C.c_double)]


class _OrcResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("n_relinearizations", C.c_int),
                ("n_rejected", C.c_int), ("final_err", C.c_double)]


class Restatement:
    """The C restatement in oracle/v3dba_oracle.c."""

    def __init__(self, path=ORC_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle restatement library missing: {path} (run make -C oracle restate)")
        self.lib = C.CDLL(path)
        L = self.lib
        P, X_ = C.POINTER(_OrcProblem), C.POINTER(_OrcParams)
        L.orc_param_length.restype = C.c_double
        L.orc_param_length.argtypes = [P, X_]
        L.orc_linearize.argtypes = [P, X_, C.c_double] + [_dp] * 5
        L.orc_cost.restype = C.c_double
        L.orc_cost.argtypes = [P, X_, C.c_double, _dp]
        L.orc_normal_blocks.restype = C.c_double
        L.orc_normal_blocks.argtypes = [P, X_, C.c_double] + [_dp] * 10
        L.orc_reduced_system.argtypes = [P, C.c_int, C.c_int, C.c_double] + [_dp] * 12
        L.orc_cholesky_solve.argtypes = [C.c_int, _dp, _dp]
        L.orc_point_update.argtypes = [P, C.c_int, C.c_int] + [_dp] * 7
        L.orc_minimize.argtypes = [P, X_, C.POINTER(_OrcOptions), C.POINTER(_OrcResult), _ip, _dp, _dp, C.c_int]
        L.orc_pcg.restype = C.c_int
        L.orc_pcg.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, C.c_double, C.c_int, _dp]
        L.orc_rodrigues.argtypes = [_dp, _dp]
        L.orc_rotations_minimize.argtypes = [C.c_int, C.c_int, _dp, _ip, _dp, C.POINTER(_OrcOptions),
                                             C.POINTER(_OrcResult), _dp, C.c_int]
        L.orc_rotations_cost.restype = C.c_double
        L.orc_rotations_cost.argtypes = [C.c_int, C.c_int, _dp, _ip, _dp]

    @staticmethod
    def _problem(scene, nonvarying=(0, 0, 0)):
        keep = (_f64(scene.meas), _i32(scene.view), _i32(scene.point))
        p = _OrcProblem(scene.model, scene.mode, scene.n_cams, scene.n_points, scene.n_obs,
                        float(scene.inlier_threshold), *nonvarying, _d(keep[0]), _i(keep[1]), _i(keep[2]))
        if getattr(scene, "rig_K", None) is not None:
            rig = (_f64(scene.rig_K), _f64(scene.rig_R), _f64(scene.rig_T), _i32(scene.sub))
            keep = keep + rig
            p.n_rig = scene.n_rig
            p.rig_K, p.rig_R, p.rig_T, p.sub = _d(rig[0]), _d(rig[1]), _d(rig[2]), _i(rig[3])
        return p, keep

    @staticmethod
    def _params(arrs):
        K, R, T, dist, X = arrs
        return _OrcParams(_d(K), _d(R), _d(T), _d(dist), _d(X))

    @staticmethod
    def cached_ar(scene):
        K = scene.K if scene.K.ndim == 2 else scene.K[0]
        return float(K[1, 1] / K[0, 0]) if K[0, 0] != 0 else 1.0

    def param_length(self, scene):
        p, keep = self._problem(scene)
        arrs = _scene_arrays(scene)
        return self.lib.orc_param_length(C.byref(p), C.byref(self._params(arrs)))

    def linearize(self, scene, params=None):
        dA, dC = scene.dims
        p, keep = self._problem(scene)
        arrs = params if params is not None else _scene_arrays(scene)
        arrs = tuple(_f64(a) for a in arrs)
        n = scene.n_obs
        e, w = np.zeros((n, 2)), np.zeros(n)
        A, B, Cm = np.zeros((n, 2, dA)), np.zeros((n, 2, 3)), np.zeros((n, 2, max(dC, 1)))
        self.lib.orc_linearize(C.byref(p), C.byref(self._params(arrs)), self.cached_ar(scene),
                               _d(e), _d(w), _d(A), _d(B), _d(Cm))
        return e, w, A, B, Cm[..., :dC]

    def cost(self, scene, params=None, weights=None):
        p, keep = self._problem(scene)
        arrs = tuple(_f64(a) for a in (params if params is not None else _scene_arrays(scene)))
        return self.lib.orc_cost(C.byref(p), C.byref(self._params(arrs)), self.cached_ar(scene),
                                 _d(_f64(weights)) if weights is not None else None)

    def normal_blocks(self, scene, params=None, nonvarying=(0, 0, 0)):
        dA, dC = scene.dims
        N, M, n = scene.n_cams, scene.n_points, scene.n_obs
        p, keep = self._problem(scene, nonvarying)
        arrs = tuple(_f64(a) for a in (params if params is not None else _scene_arrays(scene)))
        dc = max(dC, 1)
        out = dict(w=np.zeros(n), U=np.zeros((N, dA, dA)), V=np.zeros((M, 3, 3)), W=np.zeros((n, dA, 3)),
                   X=np.zeros((N, dA, dc)), Y=np.zeros((M, 3, dc)), Z=np.zeros((dc, dc)),
                   ga=np.zeros((N, dA)), gb=np.zeros((M, 3)), gc=np.zeros(dc))
        err = self.lib.orc_normal_blocks(C.byref(p), C.byref(self._params(arrs)), self.cached_ar(scene),
                                         *[_d(out[k]) for k in ("w", "U", "V", "W", "X", "Y", "Z", "ga", "gb", "gc")])
        out["X"], out["Y"], out["Z"], out["gc"] = out["X"][..., :dC], out["Y"][..., :dC], out["Z"][:dC, :dC], out["gc"][:dC]
        out["err"] = err
        return out

    def reduced_system(self, scene, blocks, lam, nonvarying=(0, 0, 0)):
        dA, dC = scene.dims
        N, M = scene.n_cams, scene.n_points
        p, keep = self._problem(scene, nonvarying)
        n = N * dA + dC
        S, rhs, Vinv = np.zeros((n, n)), np.zeros(n), np.zeros((M, 3, 3))
        dc = max(dC, 1)
        Xb = np.zeros((N, dA, dc)); Xb[..., :dC] = blocks["X"]
        Yb = np.zeros((M, 3, dc)); Yb[..., :dC] = blocks["Y"]
        Zb = np.zeros((dc, dc)); Zb[:dC, :dC] = blocks["Z"]
        gcb = np.zeros(dc); gcb[:dC] = blocks["gc"]
        # the C side indexes X/Y/Z with leading dimension dC; repack without padding
        Xp = _f64(blocks["X"]) if dC else np.zeros(1)
        Yp = _f64(blocks["Y"]) if dC else np.zeros(1)
        Zp = _f64(blocks["Z"]) if dC else np.zeros(1)
        gcp = _f64(blocks["gc"]) if dC else np.zeros(1)
        fail = self.lib.orc_reduced_system(C.byref(p), dA, dC, lam, _d(_f64(blocks["U"])), _d(_f64(blocks["V"])),
                                           _d(_f64(blocks["W"])), _d(Xp), _d(Yp), _d(Zp),
                                           _d(_f64(blocks["ga"])), _d(_f64(blocks["gb"])), _d(gcp),
                                           _d(S), _d(rhs), _d(Vinv))
        return S, rhs, Vinv, fail

    def cholesky_solve(self, S, rhs):
        S = np.array(S, dtype=np.float64, copy=True)
        x = np.array(rhs, dtype=np.float64, copy=True)
        fail = self.lib.orc_cholesky_solve(S.shape[0], _d(S), _d(x))
        return x, fail

    def minimize(self, scene, tau=1e-3, max_iterations=50, nonvarying=(0, 0, 0), lambda0=1e-3,
                 trace_cap=256, gradient_threshold=1e-10, update_threshold=1e-10):
        p, keep = self._problem(scene, nonvarying)
        arrs = _scene_arrays(scene)
        opt = _OrcOptions(tau, max_iterations, gradient_threshold, update_threshold,
                          self.param_length(scene), self.cached_ar(scene), lambda0, 2.0)
        res = _OrcResult()
        ti, tl, te = np.zeros(trace_cap, dtype=np.int32), np.zeros(trace_cap), np.zeros(trace_cap)
        rc = self.lib.orc_minimize(C.byref(p), C.byref(self._params(arrs)), C.byref(opt), C.byref(res),
                                   _i(ti), _d(tl), _d(te), trace_cap)
        if rc != 0:
            raise ValueError("oracle rejected the problem")
        n = min(res.n_relinearizations, trace_cap)
        info = dict(status=res.status, iterations=res.iterations, lambda_=opt.lambda_,
                    n_relinearizations=res.n_relinearizations, n_rejected=res.n_rejected,
                    trace_cost=te[:n].copy(), trace_lambda=tl[:n].copy(), trace_iter=ti[:n].copy())
        return arrs, info

    def pcg(self, S, b, bs, rel_tol=1e-6, max_iter=1000, Minv=None):
        x = np.zeros_like(b)
        it = self.lib.orc_pcg(S.shape[0], bs, _d(_f64(S)), _d(_f64(b)),
                              _d(_f64(Minv)) if Minv is not None else None, rel_tol, max_iter, _d(x))
        return x, it

    def rotations_minimize(self, graph, rotations=None, tau=1e-3, max_iterations=200, lambda0=1e-3,
                           gradient_threshold=1e-10, update_threshold=1e-10, trace_cap=512):
        """The restated SparseRotationOptimizer run; returns (rotations (n, 3, 3), info)."""
        R = np.array(graph.R0 if rotations is None else rotations, dtype=np.float64, copy=True)
        opt = _OrcOptions(tau, max_iterations, gradient_threshold, update_threshold, 0.0, 0.0, lambda0, 2.0)
        res = _OrcResult()
        te = np.zeros(trace_cap)
        self.lib.orc_rotations_minimize(graph.n_views, graph.n_pairs, _d(_f64(graph.rel)), _i(_i32(graph.pairs)),
                                        _d(R), C.byref(opt), C.byref(res), _d(te), trace_cap)
        n = min(res.n_relinearizations, trace_cap)
        info = dict(status=res.status, iterations=res.iterations, lambda_=opt.lambda_,
                    n_relinearizations=res.n_relinearizations, n_rejected=res.n_rejected,
                    final_err=res.final_err, trace_cost=te[:n].copy())
        return R, info

    def rotations_cost(self, graph, rotations):
        return self.lib.orc_rotations_cost(graph.n_views, graph.n_pairs, _d(_f64(graph.rel)),
                                           _i(_i32(graph.pairs)), _d(_f64(rotations)))

