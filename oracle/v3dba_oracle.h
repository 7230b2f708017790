/* TEST INFRASTRUCTURE ONLY -- the CPU oracle for the sparse LM metric bundle adjuster.
 *
 * A plain-C (C99, FP64) restatement of the reference algorithm:
 *   - residual / Huber weight / Jacobian models of V3D/include/Geometry/v3d_metricbundle.h and
 *     V3D/src/Geometry/v3d_metricbundle.cpp (Std, CommonInternals, VaryingInternals),
 *   - the block normal equations and the LM loop of V3D/src/Math/v3d_optimization.cpp:719-1250,
 *   - the parameter updates (Rodrigues, intrinsics) of v3d_metricbundle.cpp:17-50,180-212,298-358.
 * The linear step is solved by eliminating the 3x3 point blocks and factoring the dense reduced
 * camera system with a Cholesky; the reference factors the full damped normal matrix with a
 * sparse LDL^T instead (v3d_optimization.cpp:1096-1145), which is the same step algebraically.
 *
 * Only tests, the smoke check and the bench's CPU-baseline leg use this library, as a checker.
 * It is pinned against the reference optimizer compiled from its own sources (oracle/_ref).
 */
#ifndef V3DBA_ORACLE_H
#define V3DBA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_MODEL_STD = 0, ORC_MODEL_COMMON = 1, ORC_MODEL_VARYING = 2, ORC_MODEL_STEREO = 3 };
enum { ORC_TIMEOUT = 0, ORC_SMALL_UPDATE = 1, ORC_CONVERGED = 2 };

typedef struct {
  int model, mode;                 /* mode = FULL_BUNDLE_* (-1..4), ignored for STD      */
  int n_cams, n_points, n_obs;
  double inlier_threshold;
  int nnA, nnB, nnC;               /* non-varying counts (first cameras/points/globals)  */
  const double* meas;              /* n_obs*2                                            */
  const int* view;                 /* n_obs                                              */
  const int* point;                /* n_obs                                              */
  /* ORC_MODEL_STEREO (StereoMetricBundleOptimizer, V3D/include/Geometry/v3d_stereobundle.h:
   * 22-163): R/T are rig poses, K/dist unused; observation k is seen by rig camera sub[k]. */
  int n_rig;
  const double* rig_K;             /* n_rig*9                                            */
  const double* rig_R;             /* n_rig*9                                            */
  const double* rig_T;             /* n_rig*3                                            */
  const int* sub;                  /* n_obs                                              */
} orc_problem;

typedef struct {                   /* row-major, in/out                                   */
  double* K;                       /* STD/VARYING: n_cams*9;  COMMON: 9 (shared)          */
  double* R;                       /* n_cams*9                                            */
  double* T;                       /* n_cams*3                                            */
  double* dist;                    /* COMMON: 4;  VARYING: n_cams*4;  STD: unused         */
  double* X;                       /* n_points*3                                          */
} orc_params;

typedef struct {
  double tau;
  int max_iterations;
  double gradient_threshold, update_threshold;
  double param_length;             /* cached at construction (v3d_metricbundle.h:37-45)   */
  double cached_aspect_ratio;      /* COMMON: K11/K00 at construction                     */
  double lambda;                   /* in: initial lambda field; out: final lambda         */
  double nu;                       /* in/out: persistent _nu of the optimizer             */
} orc_options;

typedef struct {
  int status, iterations, n_relinearizations, n_rejected;
  double final_err;                /* sum |w e|^2 at the last relinearization              */
} orc_result;

int orc_dims(int model, int mode, int* dA, int* dC);

/* |p| as cached by the optimizer constructor: sqrt(sum_i (|T_i|^2 + 3) + sum_j |X_j|^2). */
double orc_param_length(const orc_problem* p, const orc_params* x);

/* e_k = proj - m_k, Huber weights w_k, raw Jacobians A_k (2 x dA), B_k (2 x 3), C_k (2 x dC),
 * row-major per observation.  Any output may be NULL. */
int orc_linearize(const orc_problem* p, const orc_params* x, double cached_ar,
                  double* e, double* w, double* A, double* B, double* C);

/* sum_k |w_k e_k|^2; with w == NULL the Huber weights are recomputed at x. */
double orc_cost(const orc_problem* p, const orc_params* x, double cached_ar, const double* w);

/* Weighted normal-equation blocks at x (v3d_optimization.cpp:784-979).
 * U: n_cams*dA*dA, V: n_points*9, W: n_obs*dA*3 (per observation A_k^T B_k), Xc: n_cams*dA*dC,
 * Y: n_points*3*dC, Z: dC*dC, ga: n_cams*dA, gb: n_points*3, gc: dC (gradient J^T(-w e)).
 * Blocks of fixed parameters are zero.  Outputs may be NULL except where needed.  Returns err. */
double orc_normal_blocks(const orc_problem* p, const orc_params* x, double cached_ar,
                         double* w, double* U, double* V, double* W, double* Xc, double* Y,
                         double* Z, double* ga, double* gb, double* gc);

/* Dense reduced camera system for damping lambda: S (n x n row-major, full symmetric,
 * n = n_cams*dA + dC) and rhs (n).  Fixed cameras / fixed global columns get identity rows
 * and zero rhs.  Vinv (n_points*9) receives (V_j + lambda I)^-1 (zero for fixed points). */
int orc_reduced_system(const orc_problem* p, int dA, int dC, double lambda,
                       const double* U, const double* V, const double* W, const double* Xc,
                       const double* Y, const double* Z, const double* ga, const double* gb,
                       const double* gc, double* S, double* rhs, double* Vinv);

/* In-place dense Cholesky solve of S x = rhs (row-major n x n). Returns 0, or 1 when a pivot is
 * not positive (the step fails and lambda is increased). */
int orc_cholesky_solve(int n, double* S, double* rhs);

/* Back-substitution of the point updates: db_j = Vinv_j (gb_j - sum_k W_k^T da_i(k) - Y_j dc). */
void orc_point_update(const orc_problem* p, int dA, int dC, const double* Vinv, const double* W,
                      const double* Y, const double* gb, const double* da, const double* dc,
                      double* db);

/* x <- x (+) delta (v3d_metricbundle.cpp:17-50, 180-212, 298-358). da: n_cams*dA, db: n_points*3,
 * dc: dC (may be NULL when dC == 0).  Fixed parameters are left untouched. */
void orc_apply_update(const orc_problem* p, orc_params* x, double cached_ar,
                      const double* da, const double* db, const double* dc);

void orc_rodrigues(const double omega[3], double R[9]);

/* Full LM minimize (v3d_optimization.cpp:719-1250).  x is updated in place.  The optional trace
 * (cap entries) receives (iteration, lambda, err) per relinearization. */
int orc_minimize(const orc_problem* p, orc_params* x, orc_options* opt, orc_result* res,
                 int* trace_iter, double* trace_lambda, double* trace_err, int trace_cap);

/* ---- Reduced-system PCG (no counterpart in the reference) -------------------------------
 * Block-Jacobi preconditioned conjugate gradients on the dense reduced system S x = b, with the
 * block size bs (the camera block).  Minv (nb*bs*bs, nb = n/bs) may be supplied as the
 * preconditioner; when NULL the inverse diagonal blocks of S are used.  Stops when
 * |r| <= rel_tol * |b| or after max_iter iterations; returns the iteration count. */
int orc_pcg(int n, int bs, const double* S, const double* b, const double* Minv, double rel_tol,
            int max_iter, double* x);

/* ---- Rotation averaging ---------------------------------------------------------------
 * SparseRotationOptimizer (V3D/src/Geometry/v3d_mviewutilities.cpp:470-582) minimised by the LM
 * loop above, as refineConsistentRotations (:589-611) runs it: 2*n_pairs 9-D residuals
 * e_k = R_j - R_ij R_i of pair k' = k mod n_pairs (i = pairs[2k'], j = pairs[2k'+1]); measurement
 * k < n_pairs is attached to view i with Jacobian d/domega_i of -R_ij R_i (I + [omega_i]x), the
 * second copy to view j with d/domega_j of R_j (I + [omega_j]x); no point parameters (dimension 0),
 * so the damped normal matrix is block diagonal (3x3 per view) and each block is factored by the
 * reference's sparse LDL^T in natural order.  Update R_i <- R_i Rodrigues(delta_i); |p| = sqrt(3 n).
 * rel: n_pairs*9, pairs: n_pairs*2, R: n_views*9 (in/out).  opt->max_iterations is used as given
 * (the reference sets 200).  The optional trace receives err per relinearization. */
int orc_rotations_minimize(int n_views, int n_pairs, const double* rel, const int* pairs, double* R,
                           orc_options* opt, orc_result* res, double* trace_err, int trace_cap);
/* sum over the 2*n_pairs measurements of |R_j - R_ij R_i|^2_F. */
double orc_rotations_cost(int n_views, int n_pairs, const double* rel, const int* pairs, const double* R);
#ifdef __cplusplus
}
#endif
#endif
