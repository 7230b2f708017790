/* v3dba.h -- C-ABI of the B200 sparse Levenberg-Marquardt metric bundle adjuster.
 *
 * This is the only boundary between host callers and the CUDA implementation.  It replaces
 * the reference's SparseLevenbergOptimizer / MetricBundleOptimizer family:
 *
 *   v3dba_create           <- MetricBundleOptimizerBase ctor + the three model ctors
 *                             (V3D/include/Geometry/v3d_metricbundle.h:20-46, 111-119, 168-183,
 *                              260-273); SparseLevenbergOptimizer ctor (V3D/include/Math/
 *                              v3d_optimization.h:274-291)
 *   v3dba_set_nonvarying   <- SparseLevenbergOptimizer::setNonvaryingCounts (v3d_optimization.h:295-300)
 *   v3dba_minimize         <- SparseLevenbergOptimizer::minimize (V3D/src/Math/v3d_optimization.cpp:719-1250)
 *                             with the public knobs tau / maxIterations / gradientThreshold /
 *                             updateThreshold / lambda (v3d_optimization.h:25-68, 382) and the global
 *                             optimizerVerbosenessLevel (v3d_optimization.h:23)
 *   v3dba_set_params /
 *   v3dba_get_params       <- the optimizer's in-place mutation of the caller's cameras, points,
 *                             K and distortion references (v3d_metricbundle.h:94-95, 232-233, 316)
 *   v3dba_create with
 *   V3DBA_MODEL_STEREO     <- StereoMetricBundleOptimizer (V3D/include/Geometry/v3d_stereobundle.h:
 *                              22-163, V3D/src/Geometry/v3d_stereobundle.cpp:45-67)
 *   v3dba_refine_consistent_rotations / v3dba_rotations_*
 *                          <- V3D::refineConsistentRotations and its SparseRotationOptimizer
 *                             (V3D/include/Geometry/v3d_mviewutilities.h:359-362,
 *                              V3D/src/Geometry/v3d_mviewutilities.cpp:470-611)
 *   v3dba_minimize_batched <- the sequential loop of independent triplet / submodel adjustments
 *                             (SfM/generate_triples/src/generate_triples.cpp:403-415,
 *                              SfM/generate_submodels_L1/src/generate_submodels_L1.cpp:330-337)
 *   v3dba_triplet_stage    <- the triplet stage around that adjustment: triangulation, filtering,
 *                             survival tests, BA (generate_triples.cpp:380-415)
 *
 * Conventions: plain pointers and sizes, row-major doubles, 0-based indices, no exceptions.
 * Every entry point returns an int error code (V3DBA_OK == 0).  The reference's convergence
 * outcome is reported separately in v3dba_result.status with its own codes (TIMEOUT=0,
 * SMALL_UPDATE=1, CONVERGED=2, v3d_optimization.h:16-21).
 *
 * Parameter arrays:
 *   K    : V3DBA_MODEL_STD / VARYING -> n_cameras*9 per-camera intrinsics (row-major 3x3)
 *          V3DBA_MODEL_COMMON        -> 9 (the shared K of CommonInternalsMetricBundleOptimizer)
 *   R    : n_cameras*9 world-to-camera rotations,  T : n_cameras*3 translations
 *   dist : COMMON -> 4 {k1,k2,p1,p2};  VARYING -> n_cameras*4;  STD -> unused (may be NULL)
 *   X    : n_points*3
 *   measurements : n_measurements*2 pixels;  view / point : n_measurements camera / point ids
 */
#ifndef V3DBA_H
#define V3DBA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error codes */
enum {
  V3DBA_OK = 0,
  V3DBA_ERR_INVALID_ARGUMENT = 1,   /* null pointer, bad size, bad model / mode           */
  V3DBA_ERR_INVALID_INPUT = 2,      /* index out of range, NaN / Inf in the inputs          */
  V3DBA_ERR_CUDA = 3,               /* a CUDA call failed                                   */
  V3DBA_ERR_OUT_OF_MEMORY = 4,      /* device allocation failed                            */
  V3DBA_ERR_NO_DEVICE = 5,          /* no CUDA device                                       */
  V3DBA_ERR_UNSUPPORTED = 6,        /* a configuration this library does not handle         */
  V3DBA_ERR_TIMEOUT = 7,            /* a bounded device-side wait gave up                   */
  V3DBA_ERR_NUMERICAL = 8           /* training of the learned preconditioner diverged       */
};

/* models (the optimizer classes) */
enum {
  V3DBA_MODEL_STD = 0,              /* StdMetricBundleOptimizer                             */
  V3DBA_MODEL_COMMON = 1,           /* CommonInternalsMetricBundleOptimizer                 */
  V3DBA_MODEL_VARYING = 2,          /* VaryingInternalsMetricBundleOptimizer                */
  V3DBA_MODEL_STEREO = 3            /* StereoMetricBundleOptimizer (rigid multi-camera rigs) */
};

/* FULL_BUNDLE_* modes (V3D/include/Geometry/v3d_metricbundle.h:140-148) */
enum {
  V3DBA_FULL_BUNDLE_NO_ROTATIONS = -1,
  V3DBA_FULL_BUNDLE_METRIC = 0,
  V3DBA_FULL_BUNDLE_FOCAL_LENGTH = 1,
  V3DBA_FULL_BUNDLE_FOCAL_LENGTH_PP = 2,
  V3DBA_FULL_BUNDLE_RADIAL = 3,
  V3DBA_FULL_BUNDLE_RADIAL_TANGENTIAL = 4
};

/* LM outcome (LEVENBERG_OPTIMIZER_*, V3D/include/Math/v3d_optimization.h:16-21) */
enum {
  V3DBA_STATUS_TIMEOUT = 0,
  V3DBA_STATUS_SMALL_UPDATE = 1,
  V3DBA_STATUS_CONVERGED = 2
};

/* arithmetic of the normal-equation blocks (residuals, gradient, cost and the reduced-system
 * factorisation are always FP64) */
enum {
  V3DBA_PRECISION_MIXED = 0,        /* FP32 Jacobian blocks / Schur complement (default)    */
  V3DBA_PRECISION_FP64 = 1          /* FP64 everywhere                                      */
};

/* reduced camera system solver */
enum {
  V3DBA_SOLVER_AUTO = 0,            /* dense Cholesky up to a size limit, else PCG          */
  V3DBA_SOLVER_CHOLESKY = 1,        /* tile-sparse dense FP64 Cholesky                      */
  V3DBA_SOLVER_PCG = 2              /* preconditioned conjugate gradients                  */
};

/* preconditioner of the PCG solver */
enum {
  V3DBA_PRECOND_BLOCK_JACOBI = 0,   /* inverses of the 6x6 diagonal camera blocks           */
  V3DBA_PRECOND_LEARNED = 1,        /* block-Jacobi corrected by the learned model attached with
                                       v3dba_set_precond_model; plain block-Jacobi is the
                                       fallback                                               */
  V3DBA_PRECOND_GAUGE = 2           /* block-Jacobi plus the gauge coarse space (no network)  */
};

typedef struct v3dba_problem {
  int model;                        /* V3DBA_MODEL_*                                        */
  int mode;                         /* V3DBA_FULL_BUNDLE_*, ignored for MODEL_STD           */
  int n_cameras, n_points, n_measurements;
  double inlier_threshold;          /* Huber threshold in pixels                            */
  const double* K;
  const double* R;
  const double* T;
  const double* dist;
  const double* X;
  const double* measurements;
  const int32_t* view;
  const int32_t* point;
  /* V3DBA_MODEL_STEREO only (StereoMetricBundleOptimizer, V3D/include/Geometry/
   * v3d_stereobundle.h:22-163): R / T are the poses of the n_cameras rig positions, K and dist
   * are unused (may be NULL); measurement k is seen by camera subcamera[k] of the rig, a fixed
   * pinhole camera K_l (R_l (R_i X + T_i) + T_l).  Other models ignore these fields. */
  int n_rig_cameras;
  const double* rig_K;              /* n_rig_cameras*9                                      */
  const double* rig_R;              /* n_rig_cameras*9                                      */
  const double* rig_T;              /* n_rig_cameras*3                                      */
  const int32_t* subcamera;         /* n_measurements                                       */
} v3dba_problem;

typedef struct v3dba_options {
  double tau;                       /* initial damping factor (reference default 1e-3)      */
  int max_iterations;               /* the reference leaves it uninitialised; callers set it */
  double gradient_threshold;        /* 1e-10                                                */
  double update_threshold;          /* 1e-10                                                */
  int verbosity;                    /* optimizerVerbosenessLevel semantics (0, 1, 2)         */
  int precision;                    /* V3DBA_PRECISION_*                                    */
  int solver;                       /* V3DBA_SOLVER_*                                       */
  double pcg_tolerance;             /* relative residual per LM step (PCG solver)           */
  int pcg_max_iterations;
  double stop_cost;                 /* > 0: also stop once an accepted cost <= stop_cost    */
  int mixed_escalation;             /* MIXED only: 1 (default) switches the blocks to FP64 for
                                       the rest of the call at the first rejected step or gain
                                       ratio below 0.1; 0 keeps FP32 blocks throughout         */
  int preconditioner;               /* V3DBA_PRECOND_* (PCG solver)                         */
} v3dba_options;

typedef struct v3dba_result {
  int status;                       /* V3DBA_STATUS_*                                       */
  int iterations;                   /* currentIteration on exit                             */
  int n_relinearizations;
  int n_rejected;
  double initial_cost;              /* sum |w e|^2 at the first linearisation               */
  double cost;                      /* sum |w e|^2 at the last linearisation                */
  double lambda;                    /* damping on exit                                      */
  double device_ms;                 /* device time of the call (CUDA events)                */
  int pcg_iterations;               /* total PCG iterations (PCG solver)                    */
  int reached_stop_cost;            /* 1 when stop_cost ended the call                      */
  int fp64_from_iteration;          /* MIXED: iteration at which FP64 blocks took over, or -1 */
  int pcg_fallbacks;                /* LEARNED / GAUGE: trials re-solved with plain block-Jacobi
                                       because the preconditioned solve broke down            */
} v3dba_result;

typedef struct v3dba_handle_s* v3dba_handle;

/* Fills opts with the reference defaults (tau 1e-3, maxIterations 50, thresholds 1e-10). */
void v3dba_default_options(v3dba_options* opts);

/* Copies the problem to the GPU, builds the point-major layout, the Schur block structure and
 * the symbolic factorisation of the reduced system.  |p| for the update stopping test and the
 * COMMON aspect ratio are cached here, as the reference's constructors do. */
int v3dba_create(const v3dba_problem* problem, v3dba_handle* out);
int v3dba_destroy(v3dba_handle h);

/* Fixes the first nA cameras, nB points and nC global intrinsic parameters. */
int v3dba_set_nonvarying(v3dba_handle h, int nA, int nB, int nC);

/* lambda / _nu state carried across minimize calls, as on the reference object. */
int v3dba_set_lambda(v3dba_handle h, double lambda);

int v3dba_minimize(v3dba_handle h, const v3dba_options* opts, v3dba_result* result);

/* Host <-> device parameter transfer (same layout as v3dba_problem; dist may be NULL for STD). */
int v3dba_set_params(v3dba_handle h, const double* K, const double* R, const double* T,
                     const double* dist, const double* X);
int v3dba_get_params(v3dba_handle h, double* K, double* R, double* T, double* dist, double* X);

/* Restores the parameters passed to v3dba_create (device-to-device; no host traffic) and the
 * optimizer state of a new object (lambda 1e-3, _nu 2). */
int v3dba_reset_params(v3dba_handle h);

/* sum_k |w_k e_k|^2 with Huber weights recomputed at the current device parameters. */
int v3dba_cost(v3dba_handle h, double* cost);

/* One linearisation at the current parameters, copied to the host for inspection:
 * e (n_meas*2), w (n_meas), the weighted Jacobian blocks in the caller's measurement order
 * A (n_meas*2*dA), B (n_meas*2*3), C (n_meas*2*dC) and the gradient J^T(-w e) split as
 * ga (n_cams*dA), gb (n_points*3), gc (dC).  Any output may be NULL. */
int v3dba_linearize(v3dba_handle h, int precision, double* e, double* w, double* A, double* B,
                    double* C, double* ga, double* gb, double* gc);

/* The damped reduced camera system at the current parameters for damping lambda, in FP64:
 * S (n x n, row-major, n = n_cams*dA + dC, full symmetric) and rhs (n). */
int v3dba_reduced_system(v3dba_handle h, int precision, double lambda, double* S, double* rhs);

/* Dimensions of a model / mode (dA camera block, dC global block). */
int v3dba_dims(int model, int mode, int* dA, int* dC);

/* ---- BundlePointStructure (V3D/include/Geometry/v3d_mviewutilities.h:132-205) -------------
 * The flat bundle-adjustment inputs from a reconstruction, built on the GPU.  A reconstruction
 * (vector<TriangulatedPoint>) is passed as tracks: track j (TriangulatedPoint j) has position
 * track_pos[3 j .. 3 j + 2] and the measurements track_ptr[j] .. track_ptr[j + 1] - 1, each with
 * meas_view, meas_id and the float image position meas_pos[2 m], [2 m + 1] (PointMeasurement).
 *
 * v3dba_bundle_point_structure replaces the constructor BundlePointStructure(reconstruction,
 * nRequiredMeasurements) (h:136-158): the tracks with at least n_required measurements (a
 * negative n_required keeps none, as the reference's size_t comparison does), in order, become
 * points3d, their measurements (widened to double) measurements / measurement_ids /
 * corresponding_view / corresponding_point, and xs_indices the kept tracks' indices.  The caller
 * sizes the outputs for the maxima (n_tracks points, track_ptr[n_tracks] measurements; any may
 * be NULL) and receives the counts in *n_points and *n_measurements. */
int v3dba_bundle_point_structure(int n_tracks, const int* track_ptr, const double* track_pos, const int* meas_view,
                                 const int* meas_id, const float* meas_pos, int n_required, int* n_points,
                                 int* n_measurements, double* points3d, double* measurements, int* measurement_ids,
                                 int* corresponding_view, int* corresponding_point, int* xs_indices);

/* BundlePointStructure::createPointStructure(reconstruction, createFromScratch) (h:160-197).
 * from_scratch != 0: the reconstruction becomes n_points tracks, track i at points3d[i] with the
 * measurements whose corresponding_point is i, in their order (positions narrowed to float):
 * track_ptr (n_points + 1), track_pos (3 n_points), meas_view / meas_id / meas_pos
 * (n_measurements) are outputs and n_tracks is ignored.  from_scratch == 0: the n_tracks tracks
 * keep their measurement lists (track_ptr is an input); track xs_indices[i] gets position
 * points3d[i], and the measurements of the kept tracks, in order, get the positions
 * measurements[...] one after another (meas_view, meas_id unused).  Arrays with nothing to
 * read or write (no points, no measurements, no tracks) may be NULL. */
int v3dba_create_point_structure(int from_scratch, int n_points, int n_measurements, const double* points3d,
                                 const double* measurements, const int* measurement_ids, const int* corresponding_view,
                                 const int* corresponding_point, const int* xs_indices, int n_tracks, int* track_ptr,
                                 double* track_pos, int* meas_view, int* meas_id, float* meas_pos);

/* Standalone tile-sparse FP64 Cholesky solve on the GPU of a dense SPD system (row-major n x n,
 * host memory).  Returns V3DBA_OK and *fail = 1 when a pivot is not positive. */
int v3dba_dense_cholesky_solve(int n, const double* S, const double* rhs, double* x, int* fail);

/* Benchmark support (no counterpart in the reference): the same tile Cholesky factor + solve
 * timed alone on the GPU, `reps` times from the same input; *ms receives the mean device time of
 * one factor + solve (CUDA events), x and *fail the result.  trace (may be NULL, up to trace_cap
 * entries) receives the level kernel's phase timestamps of the last repetition ((2 * levels + 2)
 * slots per cluster rank, nanoseconds), *trace_len how many, *ranks the cluster size (0 when the
 * column kernel ran).  V3DBA_CHOL_SCHEDULE=levels|steps forces either kernel. */
int v3dba_dense_cholesky_profile(int n, const double* S, const double* rhs, int reps, double* ms, double* x,
                                 int* fail, unsigned long long* trace, int trace_cap, int* trace_len, int* ranks);

/* Accuracy check support (no counterpart in the reference): evaluates on the GPU, for each of
 * the n positive x (host array), the refined reciprocal square root the tile Cholesky takes of
 * its pivots, beside CUDA's rsqrt(x): out[2 i] = refined, out[2 i + 1] = rsqrt(x). */
int v3dba_check_pivot_reciprocals(int n, const double* x, double* out);

/* Dense SPD solve that allocates nothing (no counterpart in the reference).  For callers that
 * cannot allocate device memory where they solve: a loop that reserved its GPU memory up front
 * and cannot afford cudaMalloc's implicit device synchronisation, or a host framework that owns
 * every device allocation.  S (n x n row-major, lower triangle used), rhs, x (n) and fail (one
 * int) are device buffers owned by the caller; all working memory is a fixed array compiled into
 * the library (about 0.8 MB per GPU, held until the process exits), so n must not exceed
 * V3DBA_NOALLOC_MAX_N (larger n is rejected with V3DBA_ERR_INVALID_ARGUMENT).  Calls share that
 * array: calls that overlap on the GPU race and must not be issued.  The first call on a device
 * looks up the array's device address (cached for the rest of the process) and should come before
 * any stream capture.  The work is
 * enqueued on `stream` (a cudaStream_t, NULL for the default stream); synchronise before
 * reading x or fail (1 when a pivot is not positive). */
#define V3DBA_NOALLOC_MAX_N 256
int v3dba_dense_cholesky_solve_noalloc(int n, const double* S, const double* rhs, double* x, int* fail,
                                       void* stream);

/* Batched independent problems (triplets / submodels), all of the same model and mode, solved
 * in one persistent launch.  Parameters of every problem are updated in place; results[i]
 * receives problem i's outcome. */
int v3dba_minimize_batched(const v3dba_problem* problems, int count, const v3dba_options* opts,
                           double* const* K, double* const* R, double* const* T,
                           double* const* dist, double* const* X, v3dba_result* results);

/* ---- Triplet stage (SfM/generate_triples/src/generate_triples.cpp:380-415) ----------------
 * For every view triplet, as the reference's triplet loop does after connectTracks:
 *   1. triangulateLinear of every track with the triple cameras (K = I; least squares by
 *      Householder QR, V3D/include/Geometry/v3d_mviewutilities.h:260-303);
 *   2. filterTripleModel (generate_triples.cpp:44-81): a measurement survives when
 *      f_view * |float(project(X)) - pos| < max_reproj_error (f_view the view's average focal
 *      length), a track when at least 3 of its measurements survive;
 *   3. rejection when fewer than min_points tracks survive or fewer than min_point_ratio times
 *      the track count (generate_triples.cpp:393-398);
 *   4. StdMetricBundleOptimizer on the surviving points and measurements (inlier threshold,
 *      tau, max_iterations; the reference uses 1.0, 1e-3, 5), cameras and points refined.
 * All triplets of a call run on the GPU together: one launch triangulates and filters every
 * track, one assembles the bundle problems, one persistent launch adjusts them. */
typedef struct v3dba_triplet {
  double R[27];                     /* the three cameras' rotations (row-major 3x3 each)   */
  double T[9];                      /* and translations; the intrinsics are the identity   */
  double focal[3];                  /* calibDb.getAvgFocalLength of the three views (px)   */
  int n_tracks;
  const int32_t* track_ptr;         /* [n_tracks+1] measurements of each track             */
  const int32_t* view;              /* [track_ptr[n_tracks]] triple view 0, 1 or 2         */
  const float* pos;                 /* [2*track_ptr[n_tracks]] normalised image coordinates */
} v3dba_triplet;

typedef struct v3dba_triplet_stage_options {
  double max_reproj_error;          /* MAX_REPROJECTION_ERROR_TRIPLET (pixels), default 1.0 */
  int min_points;                   /* REQUIRED_TRIPLET_POINTS, default 50                 */
  double min_point_ratio;           /* MINIMUM_TRIPLET_POINT_RATIO, default 0.5            */
  double inlier_threshold;          /* of the adjustment, default 1.0                      */
  double tau;                       /* default 1e-3                                         */
  int max_iterations;               /* default 5                                            */
} v3dba_triplet_stage_options;

enum {
  V3DBA_TRIPLET_ACCEPTED = 0,
  V3DBA_TRIPLET_TOO_FEW_POINTS = 1, /* fewer than min_points tracks survived the filter    */
  V3DBA_TRIPLET_POINTS_DROPPED = 2  /* fewer than min_point_ratio of the tracks survived    */
};

typedef struct v3dba_triplet_result {
  int verdict;                      /* V3DBA_TRIPLET_*                                      */
  int n_tracks;                     /* nPointsBefore                                        */
  int n_points;                     /* tracks that survived the filter                      */
  int status, iterations;           /* of the adjustment (accepted triplets)                */
  double cost;                      /* of the adjustment at its last linearisation          */
  double R[27], T[9];               /* cameras after the adjustment (accepted triplets)     */
} v3dba_triplet_result;

void v3dba_default_triplet_stage_options(v3dba_triplet_stage_options* opts);

/* results[t] for every triplet; X[t] (3 * n_tracks doubles, may be NULL) receives every
 * track's point: refined for the surviving tracks of accepted triplets, the linear
 * triangulation otherwise (NaN when the track's system is rank deficient); kept[t] (one byte
 * per measurement, may be NULL) is 1 for the measurements that survived the filter.
 * device_ms (may be NULL) receives the device time of the stage's kernels (CUDA events). */
int v3dba_triplet_stage(const v3dba_triplet* triplets, int count, const v3dba_triplet_stage_options* opts,
                        v3dba_triplet_result* results, double* const* X, uint8_t* const* kept, double* device_ms);

/* The same on all triplets concatenated: triplet t's cameras at R + 27 t, T + 9 t, focal + 3 t;
 * its tracks are tracks_of[t] .. tracks_of[t+1]-1 (tracks_of[0] = 0); track g's measurements are
 * track_ptr[g] .. track_ptr[g+1]-1 of view / pos (track_ptr[0] = 0, one list over all triplets).
 * Outputs per triplet (verdict, n_points, status, iterations, cost, R_out 27, T_out 9: the
 * adjustment's for accepted triplets, the inputs' cameras otherwise) and, when not NULL, X_out
 * (3 per track) and kept (1 byte per measurement) as in v3dba_triplet_stage. */
int v3dba_triplet_stage_flat(int count, const double* R, const double* T, const double* focal, const int32_t* tracks_of,
                             const int32_t* track_ptr, const int32_t* view, const float* pos,
                             const v3dba_triplet_stage_options* opts, int32_t* verdict, int32_t* n_points,
                             int32_t* status, int32_t* iterations, double* cost, double* R_out, double* T_out,
                             double* X_out, uint8_t* kept, double* device_ms);

/* Stages of one LM iteration (benchmark support; no counterpart in the reference). */
enum {
  V3DBA_STAGE_LINEARIZE = 0,        /* residuals, Huber weights, Jacobian blocks, point sums  */
  V3DBA_STAGE_CAMERA_CHUNKS = 1,    /* partial U_i, gradient, X_i per observation chunk       */
  V3DBA_STAGE_CAMERA_FINISH = 2,    /* U_i, gradient, X_i per camera                          */
  V3DBA_STAGE_RELIN_FINALIZE = 3,   /* global sums, gradient max, initial lambda              */
  V3DBA_STAGE_POINT_ELIMINATE = 4,  /* (V_j + lambda I)^-1 and W_k V_j^-1                     */
  V3DBA_STAGE_SCHUR_CHUNKS = 5,     /* partial camera-pair blocks per chunk of pairs          */
  V3DBA_STAGE_SCHUR_FINISH = 6,     /* camera-pair blocks of the reduced system               */
  V3DBA_STAGE_RHS_CHUNKS = 7,       /* partial reduced right-hand side / border               */
  V3DBA_STAGE_RHS_FINISH = 8,       /* reduced right-hand side, camera/global border          */
  V3DBA_STAGE_GLOBAL_BLOCK = 9,     /* global block                                           */
  V3DBA_STAGE_POINT_BACKSUB = 10,   /* point updates                                          */
  V3DBA_STAGE_CAMERA_UPDATE = 11,   /* camera and global updates                              */
  V3DBA_STAGE_TRIAL_COST = 12,      /* cost of the trial step with frozen weights             */
  V3DBA_STAGE_TRIAL_FINALIZE = 13,  /* step statistics                                        */
  V3DBA_STAGE_CHOLESKY = 14,        /* tile FP64 Cholesky factor + solve                      */
  V3DBA_STAGE_ZERO = 15,            /* clearing the pattern tiles of the reduced system       */
  V3DBA_NUM_STAGES = 16
};

/* Average device time (ms) of every stage over `reps` launches each, timed with CUDA events on
 * the handle's stream at the current parameters and damping 1e-3 * max diagonal.  ms receives
 * V3DBA_NUM_STAGES values.  Leaves the parameters unchanged.  (Benchmark support; no
 * counterpart in the reference.) */
int v3dba_profile_stages(v3dba_handle h, int precision, int reps, double* ms);

/* Device-resident batch of independent problems (StdMetricBundleOptimizer, at most 4 cameras
 * each; triplets and small submodels).  One persistent launch runs the full LM loop of every
 * problem, one thread block per problem at a time, largest problems first. */
typedef struct v3dba_batch_s* v3dba_batch_t;
int v3dba_batch_create(const v3dba_problem* problems, int count, v3dba_batch_t* out);
/* The same batch from flat arrays, for callers that keep all problems in one set of buffers:
 * problem p has n_cameras[p] cameras, n_points[p] points and n_measurements[p] observations;
 * K, R (9 per camera), T (3 per camera), X (3 per point), measurements (2 per observation),
 * view and point (one per observation, indices local to the problem) hold the problems one
 * after another in order.  Same checks and results as v3dba_batch_create. */
int v3dba_batch_create_flat(int count, const int* n_cameras, const int* n_points, const int* n_measurements,
                            const double* inlier_threshold, const double* K, const double* R, const double* T,
                            const double* X, const double* measurements, const int* view, const int* point,
                            v3dba_batch_t* out);
int v3dba_batch_destroy(v3dba_batch_t b);
/* results (may be NULL) receives one entry per problem; device_ms (may be NULL) the device time. */
int v3dba_batch_minimize(v3dba_batch_t b, const v3dba_options* opts, v3dba_result* results, double* device_ms);
/* Restores the parameters the batch was created with. */
int v3dba_batch_reset(v3dba_batch_t b);
/* Schedule: the first `split` problems of the size order run with `large_threads` threads per
 * block, the rest with `small_threads` (64, 128 or 256). */
int v3dba_batch_set_schedule(v3dba_batch_t b, int large_threads, int small_threads, int split);
/* Times candidate schedules on the batch itself (restoring the parameters after each) and keeps
 * the fastest; reports it when the pointers are not NULL. */
int v3dba_batch_autotune(v3dba_batch_t b, const v3dba_options* opts, int* large_threads, int* small_threads,
                         int* split);
int v3dba_batch_get_params(v3dba_batch_t b, int index, double* R, double* T, double* X);
int v3dba_batch_get_all_params(v3dba_batch_t b, double* R, double* T, double* X);

/* ---- Learned preconditioner ----------------------------------------------------------------
 * No reference counterpart: the reference factors the damped normal equations directly
 * (V3D/src/Math/v3d_optimization.cpp:1096-1145).  These entry points replace block-Jacobi in the
 * PCG reduced-camera solve by M^-1 = G^T G.  G = (I + E) C^-1, where C C^T are the Cholesky
 * factors of the 6x6 diagonal camera blocks and E is strictly block-lower on the camera
 * co-visibility pattern (the gauge coarse space, Z (Z^T S Z)^-1 Z^T with Z spanning the 7
 * similarity-gauge motions of the cameras, is a separate option).  With F the
 * normalised off-diagonal blocks of C^-1 S C^-T, each edge's block is
 * E = -c0 F + c1 (F F)|pattern + c2 (F F^T)|pattern, and a message-passing network over the
 * co-visibility graph (3 layers, hidden 64, inputs the three 6x6 blocks of every edge) predicts
 * (c0, c1, c2) - 1.  Training minimises the probe estimate of |P - I|_F^2 / n, P the normalised
 * preconditioned system, with V3DBA_PRECOND_PROBES Rademacher probes per system. */
#define V3DBA_PRECOND_PROBES 16
typedef struct v3dba_precond_model_s* v3dba_precond_model;
typedef struct v3dba_precond_set_s* v3dba_precond_set;

/* Number of float weights of the network. */
int v3dba_precond_model_size(void);
/* weights == NULL: seeded initial weights whose output layer is zero (c = 1). */
int v3dba_precond_model_create(const float* weights, uint32_t seed, v3dba_precond_model* out);
int v3dba_precond_model_destroy(v3dba_precond_model m);
int v3dba_precond_model_get_weights(v3dba_precond_model m, float* weights);
/* Attaches a model to a handle for V3DBA_PRECOND_LEARNED (NULL detaches).  The model must
 * outlive the handle's minimize() calls that use it; a model serves one call at a time. */
int v3dba_set_precond_model(v3dba_handle h, v3dba_precond_model m);

/* A device-resident set of damped reduced camera systems (6-parameter cameras only, FP64 blocks). */
int v3dba_precond_set_create(v3dba_precond_set* out);
int v3dba_precond_set_destroy(v3dba_precond_set s);
int v3dba_precond_set_count(v3dba_precond_set s);
/* Adds a system given as 6x6 blocks S_{i,l}, i <= l, row-major (rows of camera i), every
 * diagonal block present.  R (n_cameras x 9) and T (n_cameras x 3), when not NULL, are the
 * cameras the system was linearised at, for the gauge coarse space. */
int v3dba_precond_set_add_blocks(v3dba_precond_set s, int n_cameras, int n_blocks, const int32_t* blk_i,
                                 const int32_t* blk_l, const double* blocks, const double* R, const double* T);
/* Adds the handle's reduced system (FP64 blocks) at its current parameters, damped by lambda,
 * with its right-hand side and the cameras' frames for the gauge coarse space. */
int v3dba_precond_set_capture(v3dba_precond_set s, v3dba_handle h, double lambda);
int v3dba_precond_set_info(v3dba_precond_set s, int index, int* n_cameras, int* n_edges);
/* Graph and normalised inputs of system `index`: edges (a < b) with features [F, FF, FF^T]
 * (ne x 108, row-major 6x6 blocks of the lower position (b, a)), node features (N x 4) and
 * the inverse Cholesky factors of the diagonal blocks (N x 36). */
int v3dba_precond_set_features(v3dba_precond_set s, int index, int32_t* edge_a, int32_t* edge_b, float* edge_feat,
                               float* node_feat, float* cinv);
/* Probe loss of system `index` and its gradient with respect to every weight (FP32 training
 * kernels). */
int v3dba_precond_loss_grad(v3dba_precond_model m, v3dba_precond_set s, int index, uint32_t probe_seed,
                            double* loss, float* grad);
/* Network outputs c - 1 (ne x 3) of system `index`: bf16 != 0 runs the BF16 tensor-core
 * inference kernels, else the FP32 training kernels. */
int v3dba_precond_coefficients(v3dba_precond_model m, v3dba_precond_set s, int index, int bf16, float* coeffs);
/* Adam over the set for `epochs` passes in seeded order, one step per system, with probe
 * seeds drawn from `seed`; mean loss of each epoch in loss_per_epoch (may be NULL). */
int v3dba_precond_train(v3dba_precond_model m, v3dba_precond_set s, int epochs, double learning_rate, uint32_t seed,
                        double* loss_per_epoch);
/* PCG on system `index` (FP64 blocks and vectors): iterations to |r| <= tol |b| with iters[0]
 * block-Jacobi, [1] block-Jacobi + gauge space, [2] the learned factor alone, [3] the learned
 * factor + gauge space (BF16 inference).  rhs_seed == 0 solves with the system's own right-hand
 * side (the LM's reduced gradient, for captured systems), else with a seeded N(0,1) vector.
 * Entries that do not apply are -1 (no model: [2], [3]; no camera frames: [1], [3]).  A count
 * equal to max_iter means no convergence.  ms (may be NULL) receives the device time of each
 * solve in ms (its preconditioner set-up included) and, in ms[4], of the network inference. */
int v3dba_precond_pcg_iterations(v3dba_precond_model m, v3dba_precond_set s, int index, double tol, int max_iter,
                                 uint32_t rhs_seed, int* iters, double* ms);

/* The structure v3dba_create built on the device (inspection): the number of observation pairs
 * and camera-pair blocks, and, for every pointer that is not NULL, o_orig [K] (caller's index of
 * each point-major observation), c_ptr [N+1] / c_obs [K] (observations of each camera), b_i,
 * b_l [nb] / b_ptr [nb+1] (blocks (i <= l) and their pairs), pr_k, pr_m [P] (the pairs).  Replaces
 * the host-side pattern analysis of SparseLevenbergOptimizer::setupSparseJtJ
 * (V3D/src/Math/v3d_optimization.cpp:301-554). */
int v3dba_structure(v3dba_handle h, int64_t* n_pairs, int* n_blocks, int32_t* o_orig, int32_t* c_ptr, int32_t* c_obs,
                    int32_t* b_i, int32_t* b_l, int32_t* b_ptr, int32_t* pr_k, int32_t* pr_m);

/* FP64 tensor-core (DMMA) throughput of the current GPU in TFLOP/s, measured by a short kernel
 * of independent mma.sync f64 chains on every SM (benchmark support). */
int v3dba_measure_fp64_mma_peak(double* tflops);
/* Benchmark support (no counterpart in the reference): the FP64 FMA-pipe (non-tensor) throughput of
 * the current GPU in TFLOP/s, measured by a short kernel of independent FMA chains. */
int v3dba_measure_fp64_fma_peak(double* tflops);

/* FLOPs the tile Cholesky executes per factor + solve of this problem's dense reduced system
 * (64^3 GEMM tiles of its panel and trailing tasks plus the diagonal factors; benchmark
 * support). */
int v3dba_cholesky_flops(v3dba_handle h, double* flops);

/* Which tile Cholesky this problem's dense reduced system uses: *schedule = 1 for the level
 * schedule under a nested-dissection tile order (k_chol_levels), 0 for the column-by-column
 * cluster kernel (k_chol_cluster); *n_levels = its number of levels (nt for the latter), *nt =
 * the number of 64-wide tile columns (benchmark support). */
int v3dba_cholesky_schedule(v3dba_handle h, int* schedule, int* n_levels, int* nt);

/* The level schedule of the tile Cholesky for a lower-triangle tile pattern (nt x nt row-major,
 * entry (r, c) with r >= c nonzero when the tile is) and a cluster of `ranks` CTAs (2..16),
 * computed on the host with no device work:
 * order[k] = the physical tile of logical tile k (nested dissection of the tile graph, dense
 * tiles last), the number of levels, whether the solver would use it, the cost model's estimates
 * (est_us[0] level schedule, est_us[1] column-by-column, microseconds), and the packed plan
 * (*plan_len ints, written when plan_cap is large enough; offsets[14] = where each field starts:
 * phase-1 ranges, phase-1 tasks, phase-2 ranges, phase-2 tasks, task rows, task columns, task
 * input modes, task update ranges, update columns, the order with the rhs row appended,
 * back-substitution row ranges, back-substitution rows, back-substitution column ranges of
 * (level, rank), back-substitution columns).  The environment variable
 * V3DBA_CHOL_SCHEDULE=levels|steps forces either kernel (tests). */
int v3dba_tile_schedule(int nt, const uint8_t* pattern, int ranks, int* order, int* n_levels, int* uses_levels,
                        double* est_us, int* plan, int plan_cap, int* plan_len, int* offsets);

/* ---- Rotation averaging ----------------------------------------------------------------
 * V3D::refineConsistentRotations (V3D/include/Geometry/v3d_mviewutilities.h:359-362): refines
 * n_views absolute rotations from n_pairs relative rotations R_ij ~ R_j R_i^T by the
 * SparseRotationOptimizer LM (V3D/src/Geometry/v3d_mviewutilities.cpp:470-582; residuals
 * R_j - R_ij R_i, counted once per view of the pair; updates R_i <- R_i Rodrigues(delta_i);
 * maxIterations 200).  relative_rotations: n_pairs*9, view_pairs: n_pairs*2 (first, second),
 * rotations: n_views*9 (row-major; in/out).  opts may be NULL (reference defaults, 200
 * iterations); of the options only tau, max_iterations, the two thresholds, verbosity and
 * stop_cost apply.  result may be NULL; its cost fields are sum |R_j - R_ij R_i|^2_F over the
 * 2*n_pairs measurements: initial_cost at the given rotations, cost at the last relinearisation
 * (the last value the reference's verbose trace prints; at the accepted rotations when stop_cost
 * ended the call). */
int v3dba_refine_consistent_rotations(int n_views, int n_pairs, const double* relative_rotations,
                                      const int32_t* view_pairs, double* rotations, const v3dba_options* opts,
                                      v3dba_result* result);

/* The same on a device-resident problem: create uploads the graph and builds the per-view
 * measurement lists on the GPU; minimize runs the LM in one persistent launch (the _nu state
 * carries over between calls, as on the reference object); get / set transfer the rotations;
 * reset restores the rotations passed to create; cost evaluates sum |R_j - R_ij R_i|^2_F. */
typedef struct v3dba_rotations_s* v3dba_rotations;
int v3dba_rotations_create(int n_views, int n_pairs, const double* relative_rotations, const int32_t* view_pairs,
                           const double* rotations, v3dba_rotations* out);
int v3dba_rotations_destroy(v3dba_rotations h);
int v3dba_rotations_minimize(v3dba_rotations h, const v3dba_options* opts, v3dba_result* result);
int v3dba_rotations_get(v3dba_rotations h, double* rotations);
int v3dba_rotations_set(v3dba_rotations h, const double* rotations);
int v3dba_rotations_reset(v3dba_rotations h);
int v3dba_rotations_cost(v3dba_rotations h, double* cost);
/* Lanes per view (4, 8, 16 or 32) of the linearisation sweep: create picks one from the graph's
 * mean measurements per view; autotune times the sweep with each and keeps the fastest (the
 * rotations are not changed); set_group fixes it.  Results do not depend on it beyond rounding. */
int v3dba_rotations_set_group(v3dba_rotations h, int group);
int v3dba_rotations_autotune(v3dba_rotations h, int* group);

/* Kernel launches issued by this library in the calling process so far. */
uint64_t v3dba_launch_count(void);

const char* v3dba_error_string(int code);

/* Allocation-failure injection for tests (no counterpart in the reference).  With k >= 0 the
 * k-th device allocation the library requests from now on (0: the next one) fails as an
 * exhausted cudaMalloc would: the entry point that asked returns V3DBA_ERR_OUT_OF_MEMORY after
 * releasing what it holds, and later allocations succeed again.  k = -1 switches it off.
 * Process-wide; not for production use. */
int v3dba_debug_fail_allocation(long long k);

#ifdef __cplusplus
}
#endif
#endif /* V3DBA_H */
