"""ctypes binding of the C-ABI in ``include/v3dba.h`` (``_lib/libv3dba.so``).

There is no CPU fallback: when the CUDA library is missing, or no GPU is present, the calls
raise.  Build the library with ``python -m v3dsfmtoolkit_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "libv3dba.so")

OK = 0
(ERR_INVALID_ARGUMENT, ERR_INVALID_INPUT, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_NO_DEVICE, ERR_UNSUPPORTED, ERR_TIMEOUT,
 ERR_NUMERICAL) = range(1, 9)
STATUS_TIMEOUT, STATUS_SMALL_UPDATE, STATUS_CONVERGED = 0, 1, 2
MODEL_STD, MODEL_COMMON, MODEL_VARYING, MODEL_STEREO = 0, 1, 2, 3
PRECISION_MIXED, PRECISION_FP64 = 0, 1
SOLVER_AUTO, SOLVER_CHOLESKY, SOLVER_PCG = 0, 1, 2
PRECOND_BLOCK_JACOBI, PRECOND_LEARNED, PRECOND_GAUGE = 0, 1, 2
PRECOND_PROBES = 16

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)

# every symbol include/v3dba.h declares
EXPORTS = (
    "v3dba_default_options", "v3dba_create", "v3dba_destroy", "v3dba_set_nonvarying",
    "v3dba_set_lambda", "v3dba_minimize", "v3dba_set_params", "v3dba_get_params",
    "v3dba_reset_params", "v3dba_cost", "v3dba_linearize", "v3dba_reduced_system", "v3dba_dims",
    "v3dba_dense_cholesky_solve", "v3dba_minimize_batched", "v3dba_launch_count",
    "v3dba_error_string", "v3dba_profile_stages", "v3dba_batch_create", "v3dba_batch_destroy",
    "v3dba_batch_minimize", "v3dba_batch_reset", "v3dba_batch_set_schedule", "v3dba_batch_autotune",
    "v3dba_batch_get_params", "v3dba_batch_get_all_params", "v3dba_measure_fp64_mma_peak",
    "v3dba_cholesky_flops", "v3dba_dense_cholesky_solve_noalloc", "v3dba_precond_model_size",
    "v3dba_precond_model_create", "v3dba_precond_model_destroy", "v3dba_precond_model_get_weights",
    "v3dba_set_precond_model", "v3dba_precond_set_create", "v3dba_precond_set_destroy", "v3dba_precond_set_count",
    "v3dba_precond_set_add_blocks", "v3dba_precond_set_capture", "v3dba_precond_set_info",
    "v3dba_precond_set_features", "v3dba_precond_loss_grad", "v3dba_precond_coefficients", "v3dba_precond_train",
    "v3dba_precond_pcg_iterations", "v3dba_structure", "v3dba_refine_consistent_rotations",
    "v3dba_rotations_create", "v3dba_rotations_destroy", "v3dba_rotations_minimize", "v3dba_rotations_get",
    "v3dba_rotations_set", "v3dba_rotations_reset", "v3dba_rotations_cost", "v3dba_rotations_set_group",
    "v3dba_rotations_autotune", "v3dba_default_triplet_stage_options", "v3dba_triplet_stage",
    "v3dba_triplet_stage_flat", "v3dba_cholesky_schedule", "v3dba_tile_schedule", "v3dba_debug_fail_allocation",
    "v3dba_batch_create_flat", "v3dba_dense_cholesky_profile", "v3dba_check_pivot_reciprocals",
    "v3dba_bundle_point_structure", "v3dba_create_point_structure", "v3dba_measure_fp64_fma_peak",
)
STAGES = ("linearize", "camera_chunks", "camera_finish", "relin_finalize", "point_eliminate", "schur_chunks",
          "schur_finish", "rhs_chunks", "rhs_finish", "global_block", "point_backsub", "camera_update",
          "trial_cost", "trial_finalize", "cholesky", "zero")


class Problem(C.Structure):
    _fields_ = [("model", C.c_int), ("mode", C.c_int), ("n_cameras", C.c_int), ("n_points", C.c_int),
                ("n_measurements", C.c_int), ("inlier_threshold", C.c_double), ("K", _dp), ("R", _dp),
                ("T", _dp), ("dist", _dp), ("X", _dp), ("measurements", _dp), ("view", _ip), ("point", _ip),
                ("n_rig_cameras", C.c_int), ("rig_K", _dp), ("rig_R", _dp), ("rig_T", _dp), ("subcamera", _ip)]


class Options(C.Structure):
    _fields_ = [("tau", C.c_double), ("max_iterations", C.c_int), ("gradient_threshold", C.c_double),
                ("update_threshold", C.c_double), ("verbosity", C.c_int), ("precision", C.c_int),
                ("solver", C.c_int), ("pcg_tolerance", C.c_double), ("pcg_max_iterations", C.c_int),
                ("stop_cost", C.c_double), ("mixed_escalation", C.c_int), ("preconditioner", C.c_int)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("n_relinearizations", C.c_int),
                ("n_rejected", C.c_int), ("initial_cost", C.c_double), ("cost", C.c_double),
                ("lambda_", C.c_double), ("device_ms", C.c_double), ("pcg_iterations", C.c_int),
                ("reached_stop_cost", C.c_int), ("fp64_from_iteration", C.c_int), ("pcg_fallbacks", C.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Triplet(C.Structure):
    _fields_ = [("R", C.c_double * 27), ("T", C.c_double * 9), ("focal", C.c_double * 3), ("n_tracks", C.c_int),
                ("track_ptr", _ip), ("view", _ip), ("pos", C.POINTER(C.c_float))]


class TripletStageOptions(C.Structure):
    _fields_ = [("max_reproj_error", C.c_double), ("min_points", C.c_int), ("min_point_ratio", C.c_double),
                ("inlier_threshold", C.c_double), ("tau", C.c_double), ("max_iterations", C.c_int)]


class TripletResult(C.Structure):
    _fields_ = [("verdict", C.c_int), ("n_tracks", C.c_int), ("n_points", C.c_int), ("status", C.c_int),
                ("iterations", C.c_int), ("cost", C.c_double), ("R", C.c_double * 27), ("T", C.c_double * 9)]


TRIPLET_ACCEPTED, TRIPLET_TOO_FEW_POINTS, TRIPLET_POINTS_DROPPED = 0, 1, 2


class V3dbaError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        msg = _lib().v3dba_error_string(code).decode() if _LIB is not None else str(code)
        super().__init__(f"{what}: {msg} (code {code})" if what else f"{msg} (code {code})")


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA library not built: {LIB_PATH} (python -m v3dsfmtoolkit_b200.build)")
        L = C.CDLL(LIB_PATH)
        L.v3dba_default_options.argtypes = [C.POINTER(Options)]
        L.v3dba_default_options.restype = None
        L.v3dba_create.argtypes = [C.POINTER(Problem), C.POINTER(C.c_void_p)]
        L.v3dba_destroy.argtypes = [C.c_void_p]
        L.v3dba_set_nonvarying.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.v3dba_set_lambda.argtypes = [C.c_void_p, C.c_double]
        L.v3dba_minimize.argtypes = [C.c_void_p, C.POINTER(Options), C.POINTER(Result)]
        L.v3dba_set_params.argtypes = [C.c_void_p] + [_dp] * 5
        L.v3dba_get_params.argtypes = [C.c_void_p] + [_dp] * 5
        L.v3dba_reset_params.argtypes = [C.c_void_p]
        L.v3dba_cost.argtypes = [C.c_void_p, _dp]
        L.v3dba_linearize.argtypes = [C.c_void_p, C.c_int] + [_dp] * 8
        L.v3dba_reduced_system.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp]
        L.v3dba_dims.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.v3dba_dense_cholesky_solve.argtypes = [C.c_int, _dp, _dp, _dp, C.POINTER(C.c_int)]
        L.v3dba_check_pivot_reciprocals.argtypes = [C.c_int, _dp, _dp]
        _fq = C.POINTER(C.c_float)
        L.v3dba_bundle_point_structure.argtypes = [C.c_int, _ip, _dp, _ip, _ip, _fq, C.c_int, C.POINTER(C.c_int),
                                                   C.POINTER(C.c_int), _dp, _dp, _ip, _ip, _ip, _ip]
        L.v3dba_create_point_structure.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _ip, _ip, _ip, _ip, C.c_int,
                                                   _ip, _dp, _ip, _ip, _fq]
        L.v3dba_dense_cholesky_profile.argtypes = [C.c_int, _dp, _dp, C.c_int, _dp, _dp, C.POINTER(C.c_int),
                                                   C.POINTER(C.c_uint64), C.c_int, C.POINTER(C.c_int),
                                                   C.POINTER(C.c_int)]
        L.v3dba_minimize_batched.argtypes = [C.POINTER(Problem), C.c_int, C.POINTER(Options)] + \
            [C.POINTER(_dp)] * 5 + [C.POINTER(Result)]
        L.v3dba_profile_stages.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        L.v3dba_batch_create.argtypes = [C.POINTER(Problem), C.c_int, C.POINTER(C.c_void_p)]
        L.v3dba_batch_create_flat.argtypes = [C.c_int, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _ip, _ip,
                                              C.POINTER(C.c_void_p)]
        L.v3dba_batch_destroy.argtypes = [C.c_void_p]
        L.v3dba_batch_minimize.argtypes = [C.c_void_p, C.POINTER(Options), C.POINTER(Result), _dp]
        L.v3dba_batch_reset.argtypes = [C.c_void_p]
        L.v3dba_batch_set_schedule.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.v3dba_batch_autotune.argtypes = [C.c_void_p, C.POINTER(Options)] + [C.POINTER(C.c_int)] * 3
        L.v3dba_batch_get_params.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp]
        L.v3dba_batch_get_all_params.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.v3dba_measure_fp64_mma_peak.argtypes = [_dp]
        L.v3dba_measure_fp64_fma_peak.argtypes = [_dp]
        L.v3dba_cholesky_flops.argtypes = [C.c_void_p, _dp]
        L.v3dba_cholesky_schedule.argtypes = [C.c_void_p, _ip, _ip, _ip]
        L.v3dba_tile_schedule.argtypes = [C.c_int, C.POINTER(C.c_uint8), C.c_int, _ip, _ip, _ip, _dp, _ip, C.c_int,
                                          _ip, _ip]
        L.v3dba_structure.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int)] + [_ip] * 8
        _fp = C.POINTER(C.c_float)
        L.v3dba_precond_model_size.argtypes = []
        L.v3dba_precond_model_create.argtypes = [_fp, C.c_uint32, C.POINTER(C.c_void_p)]
        L.v3dba_precond_model_destroy.argtypes = [C.c_void_p]
        L.v3dba_precond_model_get_weights.argtypes = [C.c_void_p, _fp]
        L.v3dba_set_precond_model.argtypes = [C.c_void_p, C.c_void_p]
        L.v3dba_precond_set_create.argtypes = [C.POINTER(C.c_void_p)]
        L.v3dba_precond_set_destroy.argtypes = [C.c_void_p]
        L.v3dba_precond_set_count.argtypes = [C.c_void_p]
        L.v3dba_precond_set_add_blocks.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip, _dp, _dp, _dp]
        L.v3dba_precond_set_capture.argtypes = [C.c_void_p, C.c_void_p, C.c_double]
        L.v3dba_precond_set_info.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.v3dba_precond_set_features.argtypes = [C.c_void_p, C.c_int, _ip, _ip, _fp, _fp, _fp]
        L.v3dba_precond_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, _dp, _fp]
        L.v3dba_precond_coefficients.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, _fp]
        L.v3dba_precond_train.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_uint32, _dp]
        L.v3dba_precond_pcg_iterations.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_uint32,
                                                   C.POINTER(C.c_int), _dp]
        L.v3dba_refine_consistent_rotations.argtypes = [C.c_int, C.c_int, _dp, _ip, _dp, C.POINTER(Options),
                                                        C.POINTER(Result)]
        L.v3dba_rotations_create.argtypes = [C.c_int, C.c_int, _dp, _ip, _dp, C.POINTER(C.c_void_p)]
        L.v3dba_rotations_destroy.argtypes = [C.c_void_p]
        L.v3dba_rotations_minimize.argtypes = [C.c_void_p, C.POINTER(Options), C.POINTER(Result)]
        L.v3dba_rotations_get.argtypes = [C.c_void_p, _dp]
        L.v3dba_rotations_set.argtypes = [C.c_void_p, _dp]
        L.v3dba_rotations_reset.argtypes = [C.c_void_p]
        L.v3dba_rotations_cost.argtypes = [C.c_void_p, _dp]
        L.v3dba_rotations_set_group.argtypes = [C.c_void_p, C.c_int]
        L.v3dba_rotations_autotune.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.v3dba_default_triplet_stage_options.argtypes = [C.POINTER(TripletStageOptions)]
        L.v3dba_default_triplet_stage_options.restype = None
        L.v3dba_triplet_stage.argtypes = [C.POINTER(Triplet), C.c_int, C.POINTER(TripletStageOptions),
                                          C.POINTER(TripletResult), C.POINTER(_dp), C.POINTER(C.POINTER(C.c_ubyte)),
                                          _dp]
        L.v3dba_triplet_stage_flat.argtypes = [C.c_int, _dp, _dp, _dp, _ip, _ip, _ip, C.POINTER(C.c_float),
                                               C.POINTER(TripletStageOptions), _ip, _ip, _ip, _ip, _dp, _dp, _dp, _dp,
                                               C.POINTER(C.c_ubyte), _dp]
        L.v3dba_launch_count.restype = C.c_uint64
        L.v3dba_launch_count.argtypes = []
        L.v3dba_error_string.restype = C.c_char_p
        L.v3dba_error_string.argtypes = [C.c_int]
        L.v3dba_debug_fail_allocation.argtypes = [C.c_longlong]
        _LIB = L
    return _LIB


def library():
    """The loaded CDLL (raises if the library is missing)."""
    return _lib()


def check(rc, what=""):
    if rc != OK:
        raise V3dbaError(rc, what)


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def default_options(**kw) -> Options:
    o = Options()
    _lib().v3dba_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def dims(model, mode):
    a, c = C.c_int(), C.c_int()
    check(_lib().v3dba_dims(model, mode, C.byref(a), C.byref(c)), "v3dba_dims")
    return a.value, c.value


def fp64_mma_peak_tflops() -> float:
    t = C.c_double()
    check(_lib().v3dba_measure_fp64_mma_peak(C.byref(t)), "v3dba_measure_fp64_mma_peak")
    return t.value


def fp64_fma_peak_tflops() -> float:
    t = C.c_double()
    check(_lib().v3dba_measure_fp64_fma_peak(C.byref(t)), "v3dba_measure_fp64_fma_peak")
    return t.value


def launch_count() -> int:
    return int(_lib().v3dba_launch_count())


def debug_fail_allocation(k: int):
    """Makes the k-th device allocation from now on fail as an exhausted cudaMalloc would
    (tests); -1 switches the injection off."""
    check(_lib().v3dba_debug_fail_allocation(int(k)), "v3dba_debug_fail_allocation")


class Handle:
    """One problem resident on the GPU (wraps v3dba_create / v3dba_destroy)."""

    def __init__(self, model, mode, inlier_threshold, K, R, T, dist, X, measurements, view, point,
                 rig_K=None, rig_R=None, rig_T=None, subcamera=None):
        L = _lib()
        self._keep = [_f64(K), _f64(R), _f64(T), _f64(dist if dist is not None else np.zeros(4)), _f64(X),
                      _f64(measurements), np.ascontiguousarray(view, dtype=np.int32),
                      np.ascontiguousarray(point, dtype=np.int32)]
        K_, R_, T_, d_, X_, m_, v_, p_ = self._keep
        self.model, self.mode = int(model), int(mode)
        self.n_cams, self.n_points, self.n_obs = R_.size // 9, X_.size // 3, v_.size
        self.shapes = (K_.shape, R_.shape, T_.shape, d_.shape, X_.shape)
        prob = Problem(self.model, self.mode, self.n_cams, self.n_points, self.n_obs, float(inlier_threshold),
                       _d(K_), _d(R_), _d(T_), _d(d_), _d(X_), _d(m_), v_.ctypes.data_as(_ip), p_.ctypes.data_as(_ip))
        if rig_K is not None:
            rig = [_f64(rig_K), _f64(rig_R), _f64(rig_T), np.ascontiguousarray(subcamera, dtype=np.int32)]
            self._keep += rig
            prob.n_rig_cameras = rig[0].size // 9
            prob.rig_K, prob.rig_R, prob.rig_T = _d(rig[0]), _d(rig[1]), _d(rig[2])
            prob.subcamera = rig[3].ctypes.data_as(_ip)
        h = C.c_void_p()
        check(L.v3dba_create(C.byref(prob), C.byref(h)), "v3dba_create")
        self.h = h
        self.dA, self.dC = dims(self.model, self.mode)

    @classmethod
    def from_scene(cls, sc):
        return cls(sc.model, sc.mode, sc.inlier_threshold, sc.K, sc.R, sc.T, sc.dist, sc.X, sc.meas, sc.view, sc.point,
                   getattr(sc, "rig_K", None), getattr(sc, "rig_R", None), getattr(sc, "rig_T", None),
                   getattr(sc, "sub", None))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            _lib().v3dba_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_nonvarying(self, a, b, c):
        check(_lib().v3dba_set_nonvarying(self.h, a, b, c), "v3dba_set_nonvarying")

    def set_lambda(self, lam):
        check(_lib().v3dba_set_lambda(self.h, lam), "v3dba_set_lambda")

    def minimize(self, options: Options | None = None, **kw) -> Result:
        o = options if options is not None else default_options(**kw)
        if options is not None:
            for k, v in kw.items():
                setattr(o, k, v)
        r = Result()
        check(_lib().v3dba_minimize(self.h, C.byref(o), C.byref(r)), "v3dba_minimize")
        return r

    def structure(self):
        """The device-built structure: dict of o_orig, c_ptr, c_obs, b_i, b_l, b_ptr, pr_k, pr_m."""
        P, nb = C.c_int64(), C.c_int()
        L = _lib()
        check(L.v3dba_structure(self.h, C.byref(P), C.byref(nb), *([None] * 8)), "v3dba_structure")
        K, N = self.n_obs, self.n_cams
        sizes = {"o_orig": K, "c_ptr": N + 1, "c_obs": K, "b_i": nb.value, "b_l": nb.value, "b_ptr": nb.value + 1,
                 "pr_k": P.value, "pr_m": P.value}
        out = {k: np.zeros(max(v, 1), dtype=np.int32) for k, v in sizes.items()}
        check(L.v3dba_structure(self.h, None, None, *[out[k].ctypes.data_as(_ip) for k in sizes]), "v3dba_structure")
        return {k: out[k][:v] for k, v in sizes.items()}

    def set_precond_model(self, model):
        """Attaches a PrecondModel for preconditioner=PRECOND_LEARNED (kept alive by the handle)."""
        check(_lib().v3dba_set_precond_model(self.h, model.h if model is not None else None), "v3dba_set_precond_model")
        self._precond = model

    def get_params(self):
        out = [np.zeros(s) for s in self.shapes]
        check(_lib().v3dba_get_params(self.h, *[_d(a) for a in out]), "v3dba_get_params")
        return tuple(out)

    def set_params(self, K, R, T, dist, X):
        arrs = [_f64(K), _f64(R), _f64(T), _f64(dist if dist is not None else np.zeros(4)), _f64(X)]
        check(_lib().v3dba_set_params(self.h, *[_d(a) for a in arrs]), "v3dba_set_params")

    def reset_params(self):
        check(_lib().v3dba_reset_params(self.h), "v3dba_reset_params")

    def cost(self) -> float:
        c = C.c_double()
        check(_lib().v3dba_cost(self.h, C.byref(c)), "v3dba_cost")
        return c.value

    def linearize(self, precision=PRECISION_FP64):
        n, dA, dC = self.n_obs, self.dA, self.dC
        e, w = np.zeros((n, 2)), np.zeros(n)
        A, B, Cm = np.zeros((n, 2, dA)), np.zeros((n, 2, 3)), np.zeros((n, 2, max(dC, 1)))
        ga, gb, gc = np.zeros((self.n_cams, dA)), np.zeros((self.n_points, 3)), np.zeros(max(dC, 1))
        check(_lib().v3dba_linearize(self.h, precision, _d(e), _d(w), _d(A), _d(B), _d(Cm), _d(ga), _d(gb), _d(gc)),
              "v3dba_linearize")
        return dict(e=e, w=w, A=A, B=B, C=Cm[..., :dC], ga=ga, gb=gb, gc=gc[:dC])

    def profile_stages(self, precision=PRECISION_MIXED, reps=20):
        ms = np.zeros(len(STAGES))
        check(_lib().v3dba_profile_stages(self.h, precision, reps, _d(ms)), "v3dba_profile_stages")
        return dict(zip(STAGES, ms.tolist()))

    def cholesky_flops(self) -> float:
        f = C.c_double()
        check(_lib().v3dba_cholesky_flops(self.h, C.byref(f)), "v3dba_cholesky_flops")
        return f.value

    def cholesky_schedule(self):
        """("levels" | "steps", number of levels, number of tile columns) of the dense solve."""
        sch, nl, nt = C.c_int32(), C.c_int32(), C.c_int32()
        check(_lib().v3dba_cholesky_schedule(self.h, C.byref(sch), C.byref(nl), C.byref(nt)),
              "v3dba_cholesky_schedule")
        return ("levels" if sch.value else "steps"), nl.value, nt.value

    def reduced_system(self, lam, precision=PRECISION_FP64):
        n = self.n_cams * self.dA + self.dC
        S, rhs = np.zeros((n, n)), np.zeros(n)
        check(_lib().v3dba_reduced_system(self.h, precision, float(lam), _d(S), _d(rhs)), "v3dba_reduced_system")
        return S, rhs


LEVEL_PLAN_FIELDS = ("p1ptr", "p1", "p2ptr", "p2", "task_r", "task_c", "task_mode", "task_cptr", "ck", "perm",
                     "bptr", "brow", "blptr", "bcol")


def tile_schedule(pattern, ranks=16):
    """The level schedule of the tile Cholesky for a lower-triangle tile pattern (nt x nt bool) on
    a cluster of `ranks` CTAs: dict(order, n_levels, ranks, uses_levels, est_levels_us,
    est_steps_us, plan={field: int array})."""
    pat = np.ascontiguousarray(np.asarray(pattern, dtype=bool).astype(np.uint8))
    nt = pat.shape[0]
    L = _lib()
    order = np.zeros(nt, np.int32)
    nl, use, plen = C.c_int32(), C.c_int32(), C.c_int32()
    est = np.zeros(2)
    offs = np.zeros(len(LEVEL_PLAN_FIELDS), np.int32)
    u8 = pat.ctypes.data_as(C.POINTER(C.c_uint8))
    check(L.v3dba_tile_schedule(nt, u8, ranks, _i(order), C.byref(nl), C.byref(use), _d(est), None, 0,
                                C.byref(plen), _i(offs)), "v3dba_tile_schedule")
    buf = np.zeros(max(plen.value, 1), np.int32)
    check(L.v3dba_tile_schedule(nt, u8, ranks, _i(order), C.byref(nl), C.byref(use), _d(est), _i(buf), len(buf),
                                C.byref(plen), _i(offs)), "v3dba_tile_schedule")
    bounds = list(offs) + [plen.value]
    plan = {f: buf[bounds[i]:bounds[i + 1]].copy() for i, f in enumerate(LEVEL_PLAN_FIELDS)} if plen.value else {}
    return dict(order=order, n_levels=nl.value, ranks=ranks, uses_levels=bool(use.value), est_levels_us=float(est[0]),
                est_steps_us=float(est[1]), plan=plan)


def _tracks_args(tracks):
    ptr = np.ascontiguousarray(tracks["track_ptr"], dtype=np.int32)
    return (ptr, _f64(tracks["pos"]), np.ascontiguousarray(tracks["view"], dtype=np.int32),
            np.ascontiguousarray(tracks["id"], dtype=np.int32), np.ascontiguousarray(tracks["mpos"], dtype=np.float32))


def bundle_point_structure(tracks, n_required=2):
    """BundlePointStructure(reconstruction, nRequiredMeasurements) on the GPU
    (v3dba_bundle_point_structure).  tracks: dict of track_ptr (n+1), pos (n, 3), view (K), id (K),
    mpos (K, 2) float32.  Returns dict of points3d, measurements, measurement_ids,
    corresponding_view, corresponding_point, xs_indices."""
    ptr, pos, view, ids, mpos = _tracks_args(tracks)
    n, K = ptr.size - 1, int(ptr[-1])
    npts, nm = C.c_int(), C.c_int()
    pts, meas = np.zeros((max(n, 1), 3)), np.zeros((max(K, 1), 2))
    mid, cv, cp = (np.zeros(max(K, 1), np.int32) for _ in range(3))
    xs = np.zeros(max(n, 1), np.int32)
    check(_lib().v3dba_bundle_point_structure(n, _i(ptr), _d(pos), _i(view), _i(ids), _f32p(mpos), int(n_required),
                                              C.byref(npts), C.byref(nm), _d(pts), _d(meas), _i(mid), _i(cv), _i(cp),
                                              _i(xs)), "v3dba_bundle_point_structure")
    M, Kk = npts.value, nm.value
    return dict(points3d=pts[:M].copy(), measurements=meas[:Kk].copy(), measurement_ids=mid[:Kk].copy(),
                corresponding_view=cv[:Kk].copy(), corresponding_point=cp[:Kk].copy(), xs_indices=xs[:M].copy())


def create_point_structure(bps, from_scratch=True, tracks=None):
    """BundlePointStructure::createPointStructure on the GPU (v3dba_create_point_structure):
    the reconstruction as tracks (a new one from scratch, else `tracks` updated)."""
    pts, meas = _f64(bps["points3d"]).reshape(-1, 3), _f64(bps["measurements"]).reshape(-1, 2)
    M, K = pts.shape[0], meas.shape[0]
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
    mid, cv, cp, xs = i32(bps["measurement_ids"]), i32(bps["corresponding_view"]), i32(bps["corresponding_point"]), \
        i32(bps["xs_indices"])
    if from_scratch:
        ptr, pos = np.zeros(M + 1, np.int32), np.zeros((max(M, 1), 3))
        view, ids, mpos = np.zeros(max(K, 1), np.int32), np.zeros(max(K, 1), np.int32), np.zeros((max(K, 1), 2), np.float32)
        n = M
    else:
        ptr, pos, view, ids, mpos = (a.copy() for a in _tracks_args(tracks))
        n = ptr.size - 1
    check(_lib().v3dba_create_point_structure(1 if from_scratch else 0, M, K, _d(pts), _d(meas), _i(mid), _i(cv),
                                              _i(cp), _i(xs), n, _i(ptr), _d(pos), _i(view), _i(ids), _f32p(mpos)),
          "v3dba_create_point_structure")
    Kt = int(ptr[-1])
    return dict(track_ptr=ptr, pos=pos[:n].copy(), view=view[:Kt].copy(), id=ids[:Kt].copy(), mpos=mpos[:Kt].copy())


def check_pivot_reciprocals(x):
    """(n, 2) array: the tile Cholesky's refined 1/sqrt(x) and CUDA's rsqrt(x), on the GPU."""
    x = _f64(x)
    out = np.zeros((x.size, 2))
    check(_lib().v3dba_check_pivot_reciprocals(x.size, _d(x), _d(out)), "v3dba_check_pivot_reciprocals")
    return out


def dense_cholesky_profile(S, rhs, reps=20, trace_cap=4096):
    """(x, fail, ms per factor + solve, trace (levels, ranks) array or None) of the tile Cholesky
    timed alone on the GPU (v3dba_dense_cholesky_profile)."""
    S, rhs = _f64(S), _f64(rhs)
    x, fail, ms = np.zeros(S.shape[0]), C.c_int(), C.c_double()
    tr = np.zeros(trace_cap, dtype=np.uint64)
    tl, rk = C.c_int(), C.c_int()
    check(_lib().v3dba_dense_cholesky_profile(S.shape[0], _d(S), _d(rhs), reps, C.byref(ms), _d(x), C.byref(fail),
                                              tr.ctypes.data_as(C.POINTER(C.c_uint64)), trace_cap, C.byref(tl),
                                              C.byref(rk)), "v3dba_dense_cholesky_profile")
    trace = tr[:tl.value].reshape(-1, rk.value) if rk.value and tl.value else None
    return x, bool(fail.value), ms.value, trace


def dense_cholesky_solve(S, rhs):
    S = _f64(S)
    rhs = _f64(rhs)
    x = np.zeros_like(rhs)
    fail = C.c_int()
    check(_lib().v3dba_dense_cholesky_solve(S.shape[0], _d(S), _d(rhs), _d(x), C.byref(fail)),
          "v3dba_dense_cholesky_solve")
    return x, bool(fail.value)


def triplet_stage(triplets, timing=None, **kw):
    """The triplet stage (triangulation, filtering, survival tests, adjustment) of every triplet
    in one call; returns a list of dicts (verdict, n_points, status, iterations, cost, R, T, X,
    kept) in input order.  Keyword arguments override v3dba_triplet_stage_options; a dict passed
    as ``timing`` receives the device time of the stage's kernels under "device_ms"."""
    L = _lib()
    o = TripletStageOptions()
    L.v3dba_default_triplet_stage_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    n = len(triplets)
    arr = (Triplet * n)()
    keep, Xs, kepts = [], [], []
    for i, t in enumerate(triplets):
        tp = np.ascontiguousarray(t.track_ptr, dtype=np.int32)
        vw = np.ascontiguousarray(t.view, dtype=np.int32)
        ps = np.ascontiguousarray(t.pos, dtype=np.float32)
        keep += [tp, vw, ps]
        a = arr[i]
        a.R[:] = list(np.ascontiguousarray(t.R, dtype=np.float64).ravel())
        a.T[:] = list(np.ascontiguousarray(t.T, dtype=np.float64).ravel())
        a.focal[:] = list(np.asarray(t.focal, dtype=np.float64).ravel())
        a.n_tracks = t.n_tracks
        a.track_ptr, a.view = tp.ctypes.data_as(_ip), vw.ctypes.data_as(_ip)
        a.pos = ps.ctypes.data_as(C.POINTER(C.c_float))
        Xs.append(np.zeros((max(t.n_tracks, 1), 3)))
        kepts.append(np.zeros(max(int(tp[-1]), 1), dtype=np.uint8))
    res = (TripletResult * n)()
    Xp = (_dp * n)(*[x.ctypes.data_as(_dp) for x in Xs])
    Kp = (C.POINTER(C.c_ubyte) * n)(*[k.ctypes.data_as(C.POINTER(C.c_ubyte)) for k in kepts])
    ms = C.c_double()
    check(L.v3dba_triplet_stage(arr, n, C.byref(o), res, Xp, Kp, C.byref(ms)), "v3dba_triplet_stage")
    if timing is not None:
        timing["device_ms"] = ms.value
    out = []
    for i, t in enumerate(triplets):
        r = res[i]
        out.append(dict(verdict=r.verdict, n_points=r.n_points, status=r.status, iterations=r.iterations,
                        cost=r.cost, R=np.array(r.R[:]).reshape(3, 3, 3), T=np.array(r.T[:]).reshape(3, 3),
                        X=Xs[i][:t.n_tracks], kept=kepts[i][:int(t.track_ptr[-1])]))
    return out


def concat_triplets(triplets):
    """All triplets' inputs as the flat arrays of v3dba_triplet_stage_flat."""
    n = len(triplets)
    tracks_of = np.zeros(n + 1, dtype=np.int32)
    tracks_of[1:] = np.cumsum([t.n_tracks for t in triplets])
    m_of = np.zeros(n + 1, dtype=np.int64)
    m_of[1:] = np.cumsum([int(t.track_ptr[-1]) for t in triplets])
    track_ptr = np.concatenate([t.track_ptr[:-1] + m_of[i] for i, t in enumerate(triplets)] + [[m_of[-1]]])
    return dict(count=n, R=np.ascontiguousarray(np.stack([t.R for t in triplets]), dtype=np.float64),
                T=np.ascontiguousarray(np.stack([t.T for t in triplets]), dtype=np.float64),
                focal=np.ascontiguousarray(np.stack([t.focal for t in triplets]), dtype=np.float64),
                tracks_of=tracks_of, track_ptr=np.ascontiguousarray(track_ptr, dtype=np.int32),
                view=np.ascontiguousarray(np.concatenate([t.view for t in triplets]), dtype=np.int32),
                pos=np.ascontiguousarray(np.concatenate([t.pos for t in triplets]).reshape(-1, 2), dtype=np.float32))


def triplet_stage_flat(flat, timing=None, want_points=True, **kw):
    """v3dba_triplet_stage_flat on the arrays of :func:`concat_triplets`; returns a dict of flat
    outputs (verdict, n_points, status, iterations, cost, R, T per triplet; X per track and kept
    per measurement unless want_points is False)."""
    L = _lib()
    o = TripletStageOptions()
    L.v3dba_default_triplet_stage_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    n = flat["count"]
    n_trk, n_meas = int(flat["tracks_of"][-1]), int(flat["track_ptr"][-1])
    out = dict(verdict=np.zeros(n, np.int32), n_points=np.zeros(n, np.int32), status=np.zeros(n, np.int32),
               iterations=np.zeros(n, np.int32), cost=np.zeros(n), R=np.zeros((n, 3, 3, 3)), T=np.zeros((n, 3, 3)))
    if want_points:
        out["X"], out["kept"] = np.zeros((max(n_trk, 1), 3)), np.zeros(max(n_meas, 1), np.uint8)
    ms = C.c_double()
    ip = lambda a: a.ctypes.data_as(_ip)
    check(L.v3dba_triplet_stage_flat(n, _d(flat["R"]), _d(flat["T"]), _d(flat["focal"]), ip(flat["tracks_of"]),
                                     ip(flat["track_ptr"]), ip(flat["view"]),
                                     flat["pos"].ctypes.data_as(C.POINTER(C.c_float)), C.byref(o),
                                     ip(out["verdict"]), ip(out["n_points"]), ip(out["status"]), ip(out["iterations"]),
                                     _d(out["cost"]), _d(out["R"]), _d(out["T"]),
                                     _d(out["X"]) if want_points else None,
                                     out["kept"].ctypes.data_as(C.POINTER(C.c_ubyte)) if want_points else None,
                                     C.byref(ms)), "v3dba_triplet_stage_flat")
    if want_points:
        out["X"], out["kept"] = out["X"][:n_trk], out["kept"][:n_meas]
    if timing is not None:
        timing["device_ms"] = ms.value
    return out


def rotation_options(**kw) -> Options:
    """Reference defaults with SparseRotationOptimizer's maxIterations = 200."""
    o = default_options(max_iterations=200)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def refine_consistent_rotations(relative_rotations, view_pairs, rotations, options: Options | None = None, **kw):
    """V3D::refineConsistentRotations through the C-ABI: returns (refined rotations (n, 3, 3),
    Result).  ``rotations`` is not modified."""
    rel = _f64(relative_rotations).reshape(-1, 9)
    pairs = np.ascontiguousarray(view_pairs, dtype=np.int32).reshape(-1, 2)
    R = np.array(rotations, dtype=np.float64, copy=True).reshape(-1, 3, 3)
    o = options if options is not None else rotation_options(**kw)
    r = Result()
    check(_lib().v3dba_refine_consistent_rotations(R.shape[0], pairs.shape[0], _d(rel), pairs.ctypes.data_as(_ip),
                                                   _d(R), C.byref(o), C.byref(r)), "v3dba_refine_consistent_rotations")
    return R, r


class Rotations:
    """A rotation-averaging problem resident on the GPU (wraps v3dba_rotations_*)."""

    def __init__(self, relative_rotations, view_pairs, rotations):
        self._rel = _f64(relative_rotations).reshape(-1, 9)
        self._pairs = np.ascontiguousarray(view_pairs, dtype=np.int32).reshape(-1, 2)
        R0 = _f64(rotations).reshape(-1, 9)
        self.n_views, self.n_pairs = R0.shape[0], self._pairs.shape[0]
        h = C.c_void_p()
        check(_lib().v3dba_rotations_create(self.n_views, self.n_pairs, _d(self._rel), self._pairs.ctypes.data_as(_ip),
                                            _d(R0), C.byref(h)), "v3dba_rotations_create")
        self.h = h

    @classmethod
    def from_graph(cls, graph):
        return cls(graph.rel, graph.pairs, graph.R0)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            _lib().v3dba_rotations_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def minimize(self, options: Options | None = None, **kw) -> Result:
        o = options if options is not None else rotation_options(**kw)
        if options is not None:
            for k, v in kw.items():
                setattr(o, k, v)
        r = Result()
        check(_lib().v3dba_rotations_minimize(self.h, C.byref(o), C.byref(r)), "v3dba_rotations_minimize")
        return r

    def get(self):
        R = np.zeros((self.n_views, 3, 3))
        check(_lib().v3dba_rotations_get(self.h, _d(R)), "v3dba_rotations_get")
        return R

    def set(self, rotations):
        check(_lib().v3dba_rotations_set(self.h, _d(_f64(rotations))), "v3dba_rotations_set")

    def reset(self):
        check(_lib().v3dba_rotations_reset(self.h), "v3dba_rotations_reset")

    def cost(self) -> float:
        c = C.c_double()
        check(_lib().v3dba_rotations_cost(self.h, C.byref(c)), "v3dba_rotations_cost")
        return c.value

    def set_group(self, group: int):
        check(_lib().v3dba_rotations_set_group(self.h, group), "v3dba_rotations_set_group")

    def autotune(self) -> int:
        g = C.c_int()
        check(_lib().v3dba_rotations_autotune(self.h, C.byref(g)), "v3dba_rotations_autotune")
        return g.value


class Batch:
    """Many small independent problems (StdMetricBundleOptimizer, <= 4 cameras each) solved in one
    persistent launch (wraps v3dba_batch_*)."""

    def __init__(self, scenes=None, flat=None):
        L = _lib()
        if flat is not None:
            self._init_flat(L, flat)
            return
        self.scenes = list(scenes)
        self._keep = []
        probs = (Problem * len(self.scenes))()
        for i, sc in enumerate(self.scenes):
            arrs = [_f64(sc.K), _f64(sc.R), _f64(sc.T), _f64(sc.X), _f64(sc.meas),
                    np.ascontiguousarray(sc.view, dtype=np.int32), np.ascontiguousarray(sc.point, dtype=np.int32)]
            self._keep.append(arrs)
            K_, R_, T_, X_, m_, v_, p_ = arrs
            probs[i] = Problem(sc.model, sc.mode, sc.n_cams, sc.n_points, sc.n_obs, float(sc.inlier_threshold),
                               _d(K_), _d(R_), _d(T_), None, _d(X_), _d(m_), v_.ctypes.data_as(_ip), p_.ctypes.data_as(_ip))
        h = C.c_void_p()
        check(L.v3dba_batch_create(probs, len(self.scenes), C.byref(h)), "v3dba_batch_create")
        self.h = h
        self.count = len(self.scenes)

    def _init_flat(self, L, f):
        self.scenes = None
        self.flat = f
        h = C.c_void_p()
        check(L.v3dba_batch_create_flat(len(f["n_cams"]), _i(f["n_cams"]), _i(f["n_points"]), _i(f["n_obs"]),
                                        _d(f["thr"]), _d(f["K"]), _d(f["R"]), _d(f["T"]), _d(f["X"]), _d(f["meas"]),
                                        _i(f["view"]), _i(f["point"]), C.byref(h)), "v3dba_batch_create_flat")
        self.h = h
        self.count = len(f["n_cams"])

    @classmethod
    def from_flat(cls, flat):
        """A batch from the flat arrays of :func:`concat_problems` (v3dba_batch_create_flat)."""
        return cls(flat=flat)

    def get_all_params(self):
        """(R, T, X) of every problem, concatenated in problem order (v3dba_batch_get_all_params)."""
        f = self.flat if self.scenes is None else concat_problems(self.scenes)
        nc, npt = int(f["n_cams"].sum()), int(f["n_points"].sum())
        R, T, X = np.zeros((nc, 3, 3)), np.zeros((nc, 3)), np.zeros((npt, 3))
        check(_lib().v3dba_batch_get_all_params(self.h, _d(R), _d(T), _d(X)), "v3dba_batch_get_all_params")
        return R, T, X

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            _lib().v3dba_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def minimize(self, options: Options | None = None, want_results=True, **kw):
        o = options if options is not None else default_options(**kw)
        res = (Result * self.count)() if want_results else None
        ms = C.c_double()
        check(_lib().v3dba_batch_minimize(self.h, C.byref(o), res, C.byref(ms)), "v3dba_batch_minimize")
        return (list(res) if want_results else None), ms.value

    def reset(self):
        check(_lib().v3dba_batch_reset(self.h), "v3dba_batch_reset")

    def set_schedule(self, large_threads, small_threads, split):
        check(_lib().v3dba_batch_set_schedule(self.h, large_threads, small_threads, split), "v3dba_batch_set_schedule")

    def autotune(self, options: Options | None = None, **kw):
        o = options if options is not None else default_options(**kw)
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(_lib().v3dba_batch_autotune(self.h, C.byref(o), C.byref(a), C.byref(b), C.byref(c)), "v3dba_batch_autotune")
        return a.value, b.value, c.value

    def get_params(self, i):
        if self.scenes is not None:
            nc, npt = self.scenes[i].n_cams, self.scenes[i].n_points
        else:
            nc, npt = int(self.flat["n_cams"][i]), int(self.flat["n_points"][i])
        R, T, X = np.zeros((nc, 3, 3)), np.zeros((nc, 3)), np.zeros((npt, 3))
        check(_lib().v3dba_batch_get_params(self.h, i, _d(R), _d(T), _d(X)), "v3dba_batch_get_params")
        return R, T, X


def concat_problems(scenes):
    """The flat arrays v3dba_batch_create_flat takes, for a list of StdMetricBundleOptimizer scenes:
    per-problem counts and thresholds, and every problem's K, R, T, X, measurements, view and
    point one after another (indices local to each problem)."""
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
    return {
        "n_cams": i32([sc.n_cams for sc in scenes]), "n_points": i32([sc.n_points for sc in scenes]),
        "n_obs": i32([sc.n_obs for sc in scenes]),
        "thr": _f64([sc.inlier_threshold for sc in scenes]),
        "K": _f64(np.concatenate([np.reshape(sc.K, (-1, 3, 3)) for sc in scenes])),
        "R": _f64(np.concatenate([sc.R for sc in scenes])), "T": _f64(np.concatenate([sc.T for sc in scenes])),
        "X": _f64(np.concatenate([sc.X for sc in scenes])), "meas": _f64(np.concatenate([sc.meas for sc in scenes])),
        "view": i32(np.concatenate([sc.view for sc in scenes])),
        "point": i32(np.concatenate([sc.point for sc in scenes])),
    }


def _f32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None


class PrecondModel:
    """The learned preconditioner network (weights on the device)."""

    def __init__(self, weights=None, seed=0):
        self.h = C.c_void_p()
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        if w is not None and w.size != self.size():
            raise ValueError(f"expected {self.size()} weights, got {w.size}")
        check(_lib().v3dba_precond_model_create(_f32p(w), seed, C.byref(self.h)), "v3dba_precond_model_create")

    @staticmethod
    def size() -> int:
        return int(_lib().v3dba_precond_model_size())

    @classmethod
    def load(cls, path):
        return cls(np.load(path).astype(np.float32))

    def weights(self):
        w = np.zeros(self.size(), dtype=np.float32)
        check(_lib().v3dba_precond_model_get_weights(self.h, _f32p(w)), "v3dba_precond_model_get_weights")
        return w

    def close(self):
        if self.h:
            _lib().v3dba_precond_model_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def loss_grad(self, pset, index, probe_seed):
        loss = C.c_double()
        g = np.zeros(self.size(), dtype=np.float32)
        check(_lib().v3dba_precond_loss_grad(self.h, pset.h, index, probe_seed, C.byref(loss), _f32p(g)),
              "v3dba_precond_loss_grad")
        return loss.value, g

    def coefficients(self, pset, index, bf16=True):
        ne = pset.info(index)[1]
        c = np.zeros((max(ne, 1), 3), dtype=np.float32)
        check(_lib().v3dba_precond_coefficients(self.h, pset.h, index, 1 if bf16 else 0, _f32p(c)),
              "v3dba_precond_coefficients")
        return c[:ne]

    def train(self, pset, epochs, learning_rate=1e-3, seed=0):
        hist = np.zeros(max(epochs, 1))
        check(_lib().v3dba_precond_train(self.h, pset.h, epochs, learning_rate, seed, _d(hist)), "v3dba_precond_train")
        return hist[:epochs]


class PrecondSet:
    """A device-resident set of damped reduced camera systems."""

    def __init__(self):
        self.h = C.c_void_p()
        check(_lib().v3dba_precond_set_create(C.byref(self.h)), "v3dba_precond_set_create")

    def __len__(self):
        return int(_lib().v3dba_precond_set_count(self.h))

    def add_blocks(self, n_cams, blk_i, blk_l, blocks, R=None, T=None):
        bi = np.ascontiguousarray(blk_i, dtype=np.int32)
        bl = np.ascontiguousarray(blk_l, dtype=np.int32)
        b = _f64(blocks)
        R = None if R is None else _f64(R)
        T = None if T is None else _f64(T)
        check(_lib().v3dba_precond_set_add_blocks(self.h, n_cams, bi.size, bi.ctypes.data_as(_ip),
                                                  bl.ctypes.data_as(_ip), _d(b), _d(R), _d(T)),
              "v3dba_precond_set_add_blocks")

    def capture(self, handle, lam):
        check(_lib().v3dba_precond_set_capture(self.h, handle.h, lam), "v3dba_precond_set_capture")

    def info(self, index):
        n, e = C.c_int(), C.c_int()
        check(_lib().v3dba_precond_set_info(self.h, index, C.byref(n), C.byref(e)), "v3dba_precond_set_info")
        return n.value, e.value

    def features(self, index):
        N, ne = self.info(index)
        ea, eb = np.zeros(max(ne, 1), np.int32), np.zeros(max(ne, 1), np.int32)
        xe = np.zeros((max(ne, 1), 108), np.float32)
        xn, cinv = np.zeros((N, 4), np.float32), np.zeros((N, 6, 6), np.float32)
        check(_lib().v3dba_precond_set_features(self.h, index, ea.ctypes.data_as(_ip), eb.ctypes.data_as(_ip),
                                                _f32p(xe), _f32p(xn), _f32p(cinv)), "v3dba_precond_set_features")
        return ea[:ne], eb[:ne], xe[:ne], xn, cinv

    def pcg_iterations(self, index, model=None, tol=1e-6, max_iter=2000, rhs_seed=0, times=False):
        """PCG iterations of system `index`: dict with keys jacobi, jacobi_gauge, learned,
        learned_gauge (None where a variant does not apply); with times=True also the device ms
        of each solve and of the network inference."""
        it = (C.c_int * 4)()
        ms = np.zeros(5)
        check(_lib().v3dba_precond_pcg_iterations(model.h if model is not None else None, self.h, index, tol, max_iter,
                                                  rhs_seed, it, _d(ms)), "v3dba_precond_pcg_iterations")
        keys = ("jacobi", "jacobi_gauge", "learned", "learned_gauge")
        out = {k: (int(v) if v >= 0 else None) for k, v in zip(keys, it)}
        if times:
            out["ms"] = {k: (float(v) if v >= 0 else None) for k, v in zip(keys + ("inference",), ms)}
        return out

    def close(self):
        if self.h:
            _lib().v3dba_precond_set_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
