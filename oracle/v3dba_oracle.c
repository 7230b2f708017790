/* TEST INFRASTRUCTURE ONLY -- plain-C FP64 restatement of the reference's sparse LM metric
 * bundle adjustment (the oracle).  See v3dba_oracle.h for the scope; every function cites the
 * reference lines it restates.  Nothing in the product links or calls this file.
 */
#include "v3dba_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* FULL_BUNDLE_* modes (V3D/include/Geometry/v3d_metricbundle.h:140-148). */
enum { NO_ROT = -1, METRIC = 0, FOCAL = 1, FOCAL_PP = 2, RADIAL = 3, RADIAL_TAN = 4 };

static int intrinsic_dim(int mode)
{
  /* globalParamDimensionFromMode / extParamDimensionFromMode, v3d_metricbundle.h:152-164,244-256 */
  switch (mode) {
    case FOCAL: return 1;
    case FOCAL_PP: return 3;
    case RADIAL: return 5;
    case RADIAL_TAN: return 7;
    default: return 0;
  }
}

int orc_dims(int model, int mode, int* dA, int* dC)
{
  if (model == ORC_MODEL_STEREO) { *dA = 6; *dC = 0; return 0; }
  if (model < ORC_MODEL_STD || model > ORC_MODEL_VARYING) return -1;
  if (model != ORC_MODEL_STD && (mode < NO_ROT || mode > RADIAL_TAN)) return -1;
  *dA = 6 + (model == ORC_MODEL_VARYING ? intrinsic_dim(mode) : 0);
  *dC = (model == ORC_MODEL_COMMON ? intrinsic_dim(mode) : 0);
  return 0;
}

double orc_param_length(const orc_problem* p, const orc_params* x)
{
  /* MetricBundleOptimizerBase ctor, v3d_metricbundle.h:37-45; nNonvarying is 0 at that time. */
  double s = 0.0;
  for (int i = 0; i < p->n_cams; ++i) {
    const double* t = x->T + 3 * i;
    s += t[0] * t[0] + t[1] * t[1] + t[2] * t[2] + 3.0;
  }
  for (int j = 0; j < p->n_points; ++j) {
    const double* X = x->X + 3 * j;
    s += X[0] * X[0] + X[1] * X[1] + X[2] * X[2];
  }
  return sqrt(s);
}

/* ---- small dense helpers (row-major) ------------------------------------------------- */

static void matmul(const double* A, const double* B, double* C, int m, int k, int n)
{
  for (int r = 0; r < m; ++r)
    for (int c = 0; c < n; ++c) {
      double s = 0.0;
      for (int l = 0; l < k; ++l) s += A[r * k + l] * B[l * n + c];
      C[r * n + c] = s;
    }
}

static void rot_apply(const double* R, const double* X, double* out)
{
  for (int r = 0; r < 3; ++r) out[r] = R[3 * r] * X[0] + R[3 * r + 1] * X[1] + R[3 * r + 2] * X[2];
}

/* Brown distortion, V3D/include/Geometry/v3d_distortion.h:18-72. dist = {k1,k2,p1,p2}. */
static void distort(const double* d, const double* u, double* xd)
{
  double r2 = u[0] * u[0] + u[1] * u[1];
  double kr = 1.0 + d[0] * r2 + d[1] * r2 * r2;
  xd[0] = kr * u[0] + 2.0 * d[2] * u[0] * u[1] + d[3] * (r2 + 2.0 * u[0] * u[0]);
  xd[1] = kr * u[1] + 2.0 * d[3] * u[0] * u[1] + d[2] * (r2 + 2.0 * u[1] * u[1]);
}

static void distort_jac_point(const double* d, const double* u, double* J /*2x2*/)
{
  double r2 = u[0] * u[0] + u[1] * u[1];
  double kr = 1.0 + d[0] * r2 + d[1] * r2 * r2;
  double dkr = 2.0 * d[0] + 4.0 * d[1] * r2;
  J[0] = kr + u[0] * u[0] * dkr + 2.0 * d[2] * u[1] + 6.0 * d[3] * u[0];
  J[1] = u[0] * u[1] * dkr + 2.0 * d[2] * u[0] + 2.0 * d[3] * u[1];
  J[2] = J[1];
  J[3] = kr + u[1] * u[1] * dkr + 6.0 * d[2] * u[1] + 2.0 * d[3] * u[0];
}

static void distort_jac_radial(const double* u, double* J /*2x2: k1,k2*/)
{
  double r2 = u[0] * u[0] + u[1] * u[1];
  J[0] = u[0] * r2; J[1] = u[0] * r2 * r2;
  J[2] = u[1] * r2; J[3] = u[1] * r2 * r2;
}

static void distort_jac_tangential(const double* u, double* J /*2x2: p1,p2*/)
{
  double r2 = u[0] * u[0] + u[1] * u[1];
  J[0] = 2.0 * u[0] * u[1]; J[1] = r2 + 2.0 * u[0] * u[0];
  J[2] = r2 + 2.0 * u[1] * u[1]; J[3] = J[0];
}

/* Camera-space point XX = R X + T (CameraMatrix::transformPointIntoCameraSpace,
 * v3d_cameramatrix.h:227-230). */
static void to_camera(const orc_params* x, int i, int j, double* XX)
{
  const double* R = x->R + 9 * i;
  const double* T = x->T + 3 * i;
  const double* X = x->X + 3 * j;
  rot_apply(R, X, XX);
  XX[0] += T[0]; XX[1] += T[1]; XX[2] += T[2];
}

static const double* cam_K(const orc_problem* p, const orc_params* x, int i)
{
  return p->model == ORC_MODEL_COMMON ? x->K : x->K + 9 * i;
}

static const double* cam_dist(const orc_problem* p, const orc_params* x, int i)
{
  return p->model == ORC_MODEL_COMMON ? x->dist : x->dist + 4 * i;
}

/* Projection of point j into camera i:
 *   STD     : CameraMatrix::projectPoint, v3d_cameramatrix.h:184-190 (full K incl. skew, row 2)
 *   COMMON  : CommonInternals...::projectPoint, v3d_metricbundle.h:185-196 (shared K)
 *   VARYING : CameraMatrix::projectPoint(distortion, X), v3d_cameramatrix.h:192-205 */
static void project(const orc_problem* p, const orc_params* x, int i, int j, int k, double* q)
{
  double XX[3];
  to_camera(x, i, j, XX);
  if (p->model == ORC_MODEL_STEREO) {
    /* StereoMetricBundleOptimizer::evalResidual, v3d_stereobundle.h:66-80: rig space, then the
     * rig camera's projectPoint (v3d_cameramatrix.h:184-190) */
    int l = p->sub[k];
    double Y[3] = { XX[0], XX[1], XX[2] }, h[3];
    rot_apply(p->rig_R + 9 * l, Y, XX);
    for (int r = 0; r < 3; ++r) XX[r] += p->rig_T[3 * l + r];
    rot_apply(p->rig_K + 9 * l, XX, h);
    q[0] = h[0] / h[2];
    q[1] = h[1] / h[2];
    return;
  }
  const double* K = cam_K(p, x, i);
  if (p->model == ORC_MODEL_STD) {
    double h[3];
    rot_apply(K, XX, h);
    q[0] = h[0] / h[2];
    q[1] = h[1] / h[2];
  } else {
    double u[2] = { XX[0] / XX[2], XX[1] / XX[2] }, d[2];
    distort(cam_dist(p, x, i), u, d);
    q[0] = K[0] * d[0] + K[1] * d[1] + K[2];
    q[1] = K[4] * d[1] + K[5];
  }
}

/* Jacobians of observation k (raw, unweighted), v3d_metricbundle.cpp:52-178, 216-296.
 * A: 2 x dA, B: 2 x 3, C: 2 x dC, row-major. */
static void jacobians(const orc_problem* p, const orc_params* x, double cached_ar, int dA, int dC,
                      int i, int j, int k, double* A, double* B, double* C)
{
  const double* R = x->R + 9 * i;
  const double* T = x->T + 3 * i;
  double XX[3];
  to_camera(x, i, j, XX);

  if (p->model == ORC_MODEL_STEREO) {
    /* poseDerivatives + StereoMetricBundleOptimizer::fillJacobians, v3d_stereobundle.cpp:11-67:
     * dY/d(T, omega) = [ I | -[R X]_x ], then through the rig camera's rotation R_l; f and the
     * aspect ratio of K_l (skew and principal point ignored). */
    int l = p->sub[k];
    const double* Rl = p->rig_R + 9 * l;
    const double* Kl = p->rig_K + 9 * l;
    double RX[3] = { XX[0] - T[0], XX[1] - T[1], XX[2] - T[2] };
    double dY[18];
    memset(dY, 0, sizeof(dY));
    dY[0 * 6 + 0] = dY[1 * 6 + 1] = dY[2 * 6 + 2] = 1.0;
    dY[0 * 6 + 3] = 0.0;    dY[0 * 6 + 4] = RX[2];  dY[0 * 6 + 5] = -RX[1];
    dY[1 * 6 + 3] = -RX[2]; dY[1 * 6 + 4] = 0.0;    dY[1 * 6 + 5] = RX[0];
    dY[2 * 6 + 3] = RX[1];  dY[2 * 6 + 4] = -RX[0]; dY[2 * 6 + 5] = 0.0;
    double Xl[3], d_dRT[18], d_dX[9], dp[6];
    rot_apply(Rl, XX, Xl);
    for (int r = 0; r < 3; ++r) Xl[r] += p->rig_T[3 * l + r];
    matmul(Rl, dY, d_dRT, 3, 3, 6);
    matmul(Rl, R, d_dX, 3, 3, 3);
    double f = Kl[0], ar = Kl[4] / Kl[0];
    double bx = f / (Xl[2] * Xl[2]), by = ar * bx;
    dp[0] = bx * Xl[2]; dp[1] = 0.0;        dp[2] = -bx * Xl[0];
    dp[3] = 0.0;        dp[4] = by * Xl[2]; dp[5] = -by * Xl[1];
    matmul(dp, d_dRT, A, 2, 3, 6);
    matmul(dp, d_dX, B, 2, 3, 3);
    (void)cached_ar; (void)dA; (void)dC; (void)C;
    return;
  }

  /* poseDerivatives, v3d_metricbundle.cpp:52-71: d XX / d(T, omega) = [ I | -[XX - T]_x ],
   * d XX / d X = R. */
  double RX[3] = { XX[0] - T[0], XX[1] - T[1], XX[2] - T[2] };
  double dRT[18];
  memset(dRT, 0, sizeof(dRT));
  dRT[0 * 6 + 0] = dRT[1 * 6 + 1] = dRT[2 * 6 + 2] = 1.0;
  /* -[v]_x  with v = RX */
  dRT[0 * 6 + 3] = 0.0;    dRT[0 * 6 + 4] = RX[2];  dRT[0 * 6 + 5] = -RX[1];
  dRT[1 * 6 + 3] = -RX[2]; dRT[1 * 6 + 4] = 0.0;    dRT[1 * 6 + 5] = RX[0];
  dRT[2 * 6 + 3] = RX[1];  dRT[2 * 6 + 4] = -RX[0]; dRT[2 * 6 + 5] = 0.0;

  const double* K = cam_K(p, x, i);
  double dp_dXX[6];

  if (p->model == ORC_MODEL_STD) {
    /* StdMetricBundleOptimizer::fillJacobians, v3d_metricbundle.cpp:76-98: skew and principal
     * point are ignored; ar = K11/K00. */
    double f = K[0], ar = K[4] / K[0];
    double bx = f / (XX[2] * XX[2]), by = ar * bx;
    dp_dXX[0] = bx * XX[2]; dp_dXX[1] = 0.0;        dp_dXX[2] = -bx * XX[0];
    dp_dXX[3] = 0.0;        dp_dXX[4] = by * XX[2]; dp_dXX[5] = -by * XX[1];
    matmul(dp_dXX, dRT, A, 2, 3, 6);
    matmul(dp_dXX, R, B, 2, 3, 3);
    return;
  }

  /* CommonInternals (v3d_metricbundle.cpp:102-178) / VaryingInternals (:216-296). */
  int mode = p->mode;
  if (mode == NO_ROT) {
    /* Q4: zeroes the first three columns of dXX/dRT, which are the translation columns. */
    for (int r = 0; r < 3; ++r) dRT[r * 6 + 0] = dRT[r * 6 + 1] = dRT[r * 6 + 2] = 0.0;
  }
  const double* dist = cam_dist(p, x, i);
  double f, ar;
  if (p->model == ORC_MODEL_COMMON) { f = K[0]; ar = cached_ar; }
  else { f = K[0]; ar = K[4] / K[0]; }

  double u[2] = { XX[0] / XX[2], XX[1] / XX[2] }, xd[2];
  distort(dist, u, xd);
  double fx = f, fy = ar * f;      /* dp/dxd = diag(fx, fy) */
  double dxu_dXX[6] = { 1.0 / XX[2], 0.0, -XX[0] / (XX[2] * XX[2]),
                        0.0, 1.0 / XX[2], -XX[1] / (XX[2] * XX[2]) };
  double Jd[4];
  distort_jac_point(dist, u, Jd);
  double dp_dxu[4] = { fx * Jd[0], fx * Jd[1], fy * Jd[2], fy * Jd[3] };
  matmul(dp_dxu, dxu_dXX, dp_dXX, 2, 2, 3);

  double Apose[12];
  matmul(dp_dXX, dRT, Apose, 2, 3, 6);
  matmul(dp_dXX, R, B, 2, 3, 3);
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 6; ++c) A[r * dA + c] = Apose[r * 6 + c];

  /* Intrinsic columns [f, cx, cy, k1, k2, p1, p2] (mode fall-through, :147-177 / :265-295).
   * For COMMON they form C; for VARYING they are appended to A at column 6. */
  double* G = (p->model == ORC_MODEL_COMMON) ? C : A + 6;
  int ld = (p->model == ORC_MODEL_COMMON) ? dC : dA;
  int nint = intrinsic_dim(mode);
  if (nint >= 7) {
    double Jt[4];
    distort_jac_tangential(u, Jt);
    G[0 * ld + 5] = fx * Jt[0]; G[0 * ld + 6] = fx * Jt[1];
    G[1 * ld + 5] = fy * Jt[2]; G[1 * ld + 6] = fy * Jt[3];
  }
  if (nint >= 5) {
    double Jr[4];
    distort_jac_radial(u, Jr);
    G[0 * ld + 3] = fx * Jr[0]; G[0 * ld + 4] = fx * Jr[1];
    G[1 * ld + 3] = fy * Jr[2]; G[1 * ld + 4] = fy * Jr[3];
  }
  if (nint >= 3) {
    G[0 * ld + 1] = 1.0; G[0 * ld + 2] = 0.0;
    G[1 * ld + 1] = 0.0; G[1 * ld + 2] = 1.0;
  }
  if (nint >= 1) {
    /* Q5: d/df uses xd on both rows (the aspect ratio is ignored). */
    G[0 * ld + 0] = xd[0];
    G[1 * ld + 0] = xd[1];
  }
}

static double huber_weight(double thr, const double* e)
{
  /* MetricBundleOptimizerBase::fillWeights, v3d_metricbundle.h:49-57 */
  double n = sqrt(e[0] * e[0] + e[1] * e[1]);
  return (n < thr) ? 1.0 : sqrt(thr / n);
}

int orc_linearize(const orc_problem* p, const orc_params* x, double cached_ar,
                  double* e, double* w, double* A, double* B, double* C)
{
  int dA, dC;
  if (orc_dims(p->model, p->mode, &dA, &dC)) return -1;
  double a[2 * 13], b[6], c[2 * 7];
  for (int k = 0; k < p->n_obs; ++k) {
    int i = p->view[k], j = p->point[k];
    double q[2], ek[2];
    project(p, x, i, j, k, q);
    ek[0] = q[0] - p->meas[2 * k];
    ek[1] = q[1] - p->meas[2 * k + 1];
    if (e) { e[2 * k] = ek[0]; e[2 * k + 1] = ek[1]; }
    if (w) w[k] = huber_weight(p->inlier_threshold, ek);
    if (A || B || C) {
      memset(a, 0, sizeof(a)); memset(c, 0, sizeof(c));
      jacobians(p, x, cached_ar, dA, dC, i, j, k, a, b, c);
      if (A) memcpy(A + (size_t)k * 2 * dA, a, sizeof(double) * 2 * dA);
      if (B) memcpy(B + (size_t)k * 6, b, sizeof(double) * 6);
      if (C && dC) memcpy(C + (size_t)k * 2 * dC, c, sizeof(double) * 2 * dC);
    }
  }
  return 0;
}

double orc_cost(const orc_problem* p, const orc_params* x, double cached_ar, const double* w)
{
  (void)cached_ar;
  double err = 0.0;
  for (int k = 0; k < p->n_obs; ++k) {
    double q[2], ek[2];
    project(p, x, p->view[k], p->point[k], k, q);
    ek[0] = q[0] - p->meas[2 * k];
    ek[1] = q[1] - p->meas[2 * k + 1];
    double wk = w ? w[k] : huber_weight(p->inlier_threshold, ek);
    err += wk * wk * (ek[0] * ek[0] + ek[1] * ek[1]);
  }
  return err;
}

/* v3d_optimization.cpp:784-979: residuals scaled by w and negated, Jacobians scaled by w
 * (fillAllJacobians, v3d_optimization.h:318-362), then J^T e and the U/V/W/X/Y/Z blocks. */
double orc_normal_blocks(const orc_problem* p, const orc_params* x, double cached_ar,
                         double* w, double* U, double* V, double* W, double* Xc, double* Y,
                         double* Z, double* ga, double* gb, double* gc)
{
  int dA, dC;
  orc_dims(p->model, p->mode, &dA, &dC);
  int N = p->n_cams, M = p->n_points;
  if (U) memset(U, 0, sizeof(double) * N * dA * dA);
  if (V) memset(V, 0, sizeof(double) * M * 9);
  if (Xc && dC) memset(Xc, 0, sizeof(double) * N * dA * dC);
  if (Y && dC) memset(Y, 0, sizeof(double) * M * 3 * dC);
  if (Z && dC) memset(Z, 0, sizeof(double) * dC * dC);
  if (ga) memset(ga, 0, sizeof(double) * N * dA);
  if (gb) memset(gb, 0, sizeof(double) * M * 3);
  if (gc && dC) memset(gc, 0, sizeof(double) * dC);

  double err = 0.0;
  double a[2 * 13], b[6], c[2 * 7];
  for (int k = 0; k < p->n_obs; ++k) {
    int i = p->view[k], j = p->point[k];
    double q[2], ek[2];
    project(p, x, i, j, k, q);
    ek[0] = q[0] - p->meas[2 * k];
    ek[1] = q[1] - p->meas[2 * k + 1];
    double wk = huber_weight(p->inlier_threshold, ek);
    if (w) w[k] = wk;
    err += wk * wk * (ek[0] * ek[0] + ek[1] * ek[1]);
    double r[2] = { -wk * ek[0], -wk * ek[1] };

    int fixA = i < p->nnA, fixB = j < p->nnB;
    memset(a, 0, sizeof(a)); memset(b, 0, sizeof(b)); memset(c, 0, sizeof(c));
    /* An observation whose camera and point are both fixed still constrains the globals
     * (the reference skips it and leaves stale Jacobians, quirk Q6). */
    jacobians(p, x, cached_ar, dA, dC, i, j, k, a, b, c);
    if (fixA) memset(a, 0, sizeof(a));
    if (fixB) memset(b, 0, sizeof(b));
    for (int l = 0; l < p->nnC && l < dC; ++l) c[l] = c[dC + l] = 0.0;
    for (int t = 0; t < 2 * dA; ++t) a[t] *= wk;
    for (int t = 0; t < 6; ++t) b[t] *= wk;
    for (int t = 0; t < 2 * dC; ++t) c[t] *= wk;

    if (!fixA) {
      if (ga) for (int l = 0; l < dA; ++l) ga[i * dA + l] += a[l] * r[0] + a[dA + l] * r[1];
      if (U)
        for (int r1 = 0; r1 < dA; ++r1)
          for (int c1 = 0; c1 < dA; ++c1)
            U[(size_t)i * dA * dA + r1 * dA + c1] += a[r1] * a[c1] + a[dA + r1] * a[dA + c1];
      if (Xc && dC)
        for (int r1 = 0; r1 < dA; ++r1)
          for (int c1 = 0; c1 < dC; ++c1)
            Xc[(size_t)i * dA * dC + r1 * dC + c1] += a[r1] * c[c1] + a[dA + r1] * c[dC + c1];
    }
    if (!fixB) {
      if (gb) for (int l = 0; l < 3; ++l) gb[j * 3 + l] += b[l] * r[0] + b[3 + l] * r[1];
      if (V)
        for (int r1 = 0; r1 < 3; ++r1)
          for (int c1 = 0; c1 < 3; ++c1)
            V[(size_t)j * 9 + r1 * 3 + c1] += b[r1] * b[c1] + b[3 + r1] * b[3 + c1];
      if (Y && dC)
        for (int r1 = 0; r1 < 3; ++r1)
          for (int c1 = 0; c1 < dC; ++c1)
            Y[(size_t)j * 3 * dC + r1 * dC + c1] += b[r1] * c[c1] + b[3 + r1] * c[dC + c1];
    }
    if (W)
      for (int r1 = 0; r1 < dA; ++r1)
        for (int c1 = 0; c1 < 3; ++c1)
          W[(size_t)k * dA * 3 + r1 * 3 + c1] = a[r1] * b[c1] + a[dA + r1] * b[3 + c1];
    if (dC) {
      if (gc) for (int l = 0; l < dC; ++l) gc[l] += c[l] * r[0] + c[dC + l] * r[1];
      if (Z)
        for (int r1 = 0; r1 < dC; ++r1)
          for (int c1 = 0; c1 < dC; ++c1) Z[r1 * dC + c1] += c[r1] * c[c1] + c[dC + r1] * c[dC + c1];
    }
  }
  return err;
}

static int inv3_sym(const double* A, double* Ai)
{
  double c00 = A[4] * A[8] - A[5] * A[7];
  double c01 = A[5] * A[6] - A[3] * A[8];
  double c02 = A[3] * A[7] - A[4] * A[6];
  double det = A[0] * c00 + A[1] * c01 + A[2] * c02;
  if (!(det != 0.0)) return 1;
  double id = 1.0 / det;
  Ai[0] = c00 * id;
  Ai[1] = (A[2] * A[7] - A[1] * A[8]) * id;
  Ai[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  Ai[3] = c01 * id;
  Ai[4] = (A[0] * A[8] - A[2] * A[6]) * id;
  Ai[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  Ai[6] = c02 * id;
  Ai[7] = (A[1] * A[6] - A[0] * A[7]) * id;
  Ai[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  return 0;
}

/* The damped system of v3d_optimization.cpp:1055-1092 with the point blocks eliminated. */
int orc_reduced_system(const orc_problem* p, int dA, int dC, double lambda,
                       const double* U, const double* V, const double* W, const double* Xc,
                       const double* Y, const double* Z, const double* ga, const double* gb,
                       const double* gc, double* S, double* rhs, double* Vinv)
{
  int N = p->n_cams, M = p->n_points;
  int n = N * dA + dC, c0 = N * dA;
  memset(S, 0, sizeof(double) * (size_t)n * n);
  memset(rhs, 0, sizeof(double) * n);

  for (int i = 0; i < N; ++i) {
    int o = i * dA;
    if (i < p->nnA) {
      for (int l = 0; l < dA; ++l) S[(size_t)(o + l) * n + o + l] = 1.0;
      continue;
    }
    for (int r = 0; r < dA; ++r) {
      rhs[o + r] = ga[i * dA + r];
      for (int c = 0; c < dA; ++c) S[(size_t)(o + r) * n + o + c] = U[(size_t)i * dA * dA + r * dA + c];
      S[(size_t)(o + r) * n + o + r] += lambda;
      for (int c = 0; c < dC; ++c) {
        double v = Xc[(size_t)i * dA * dC + r * dC + c];
        if (c < p->nnC) v = 0.0;
        S[(size_t)(o + r) * n + c0 + c] = v;
        S[(size_t)(c0 + c) * n + o + r] = v;
      }
    }
  }
  for (int r = 0; r < dC; ++r) {
    if (r < p->nnC) { S[(size_t)(c0 + r) * n + c0 + r] = 1.0; continue; }
    rhs[c0 + r] = gc[r];
    for (int c = p->nnC; c < dC; ++c) S[(size_t)(c0 + r) * n + c0 + c] = Z[r * dC + c];
    S[(size_t)(c0 + r) * n + c0 + r] += lambda;
  }

  /* observations grouped by point (any order) */
  int* cnt = (int*)calloc(M + 1, sizeof(int));
  int* idx = (int*)malloc(sizeof(int) * (p->n_obs > 0 ? p->n_obs : 1));
  for (int k = 0; k < p->n_obs; ++k) cnt[p->point[k] + 1]++;
  for (int j = 0; j < M; ++j) cnt[j + 1] += cnt[j];
  int* fill = (int*)malloc(sizeof(int) * (M + 1));
  memcpy(fill, cnt, sizeof(int) * (M + 1));
  for (int k = 0; k < p->n_obs; ++k) idx[fill[p->point[k]]++] = k;
  free(fill);

  double* T = (double*)malloc(sizeof(double) * 13 * 3 * 64);
  int fail = 0;
  for (int j = 0; j < M; ++j) {
    double* Vi = Vinv + 9 * (size_t)j;
    if (j < p->nnB) { memset(Vi, 0, 9 * sizeof(double)); continue; }
    double Vd[9];
    memcpy(Vd, V + 9 * (size_t)j, sizeof(Vd));
    Vd[0] += lambda; Vd[4] += lambda; Vd[8] += lambda;
    if (inv3_sym(Vd, Vi)) { fail = 1; memset(Vi, 0, 9 * sizeof(double)); continue; }
    int beg = cnt[j], end = cnt[j + 1], len = end - beg;
    if (len > 64) T = (double*)realloc(T, sizeof(double) * 13 * 3 * len);
    double q[3], YV[3 * 7];
    matmul(Vi, gb + 3 * (size_t)j, q, 3, 3, 1);
    if (dC) matmul(Vi, Y + (size_t)j * 3 * dC, YV, 3, 3, dC);  /* Vinv Y_j */
    for (int t = 0; t < len; ++t) matmul(W + (size_t)idx[beg + t] * dA * 3, Vi, T + t * dA * 3, dA, 3, 3);
    for (int t = 0; t < len; ++t) {
      int k = idx[beg + t], ik = p->view[k];
      if (ik < p->nnA) continue;
      const double* Tk = T + t * dA * 3;
      /* rhs_a -= W_k Vinv gb_j */
      for (int r = 0; r < dA; ++r)
        rhs[ik * dA + r] -= Tk[r * 3] * gb[3 * j] + Tk[r * 3 + 1] * gb[3 * j + 1] + Tk[r * 3 + 2] * gb[3 * j + 2];
      for (int u = 0; u < len; ++u) {
        int m = idx[beg + u], im = p->view[m];
        if (im < p->nnA) continue;
        const double* Wm = W + (size_t)m * dA * 3;
        for (int r = 0; r < dA; ++r)
          for (int c = 0; c < dA; ++c)
            S[(size_t)(ik * dA + r) * n + im * dA + c] -=
                Tk[r * 3] * Wm[c * 3] + Tk[r * 3 + 1] * Wm[c * 3 + 1] + Tk[r * 3 + 2] * Wm[c * 3 + 2];
      }
      /* camera/global border: -W_k Vinv Y_j */
      for (int r = 0; r < dA; ++r)
        for (int c = p->nnC; c < dC; ++c) {
          double v = Tk[r * 3] * Y[(size_t)j * 3 * dC + c] + Tk[r * 3 + 1] * Y[(size_t)j * 3 * dC + dC + c] +
                     Tk[r * 3 + 2] * Y[(size_t)j * 3 * dC + 2 * dC + c];
          S[(size_t)(ik * dA + r) * n + c0 + c] -= v;
          S[(size_t)(c0 + c) * n + ik * dA + r] -= v;
        }
    }
    for (int r = p->nnC; r < dC; ++r) {
      /* rhs_c -= Y_j^T Vinv gb_j ;  S_cc -= Y_j^T Vinv Y_j */
      const double* Yj = Y + (size_t)j * 3 * dC;
      rhs[c0 + r] -= Yj[r] * q[0] + Yj[dC + r] * q[1] + Yj[2 * dC + r] * q[2];
      for (int c = p->nnC; c < dC; ++c)
        S[(size_t)(c0 + r) * n + c0 + c] -= Yj[r] * YV[c] + Yj[dC + r] * YV[dC + c] + Yj[2 * dC + r] * YV[2 * dC + c];
    }
  }
  free(T); free(idx); free(cnt);
  return fail;
}

int orc_cholesky_solve(int n, double* S, double* rhs)
{
  /* Right-looking dense Cholesky S = L L^T (lower part of S overwritten by L). */
  for (int k = 0; k < n; ++k) {
    double d = S[(size_t)k * n + k];
    for (int l = 0; l < k; ++l) d -= S[(size_t)k * n + l] * S[(size_t)k * n + l];
    if (!(d > 0.0)) return 1;
    d = sqrt(d);
    S[(size_t)k * n + k] = d;
    for (int r = k + 1; r < n; ++r) {
      double s = S[(size_t)r * n + k];
      for (int l = 0; l < k; ++l) s -= S[(size_t)r * n + l] * S[(size_t)k * n + l];
      S[(size_t)r * n + k] = s / d;
    }
  }
  for (int r = 0; r < n; ++r) {
    double s = rhs[r];
    for (int l = 0; l < r; ++l) s -= S[(size_t)r * n + l] * rhs[l];
    rhs[r] = s / S[(size_t)r * n + r];
  }
  for (int r = n - 1; r >= 0; --r) {
    double s = rhs[r];
    for (int l = r + 1; l < n; ++l) s -= S[(size_t)l * n + r] * rhs[l];
    rhs[r] = s / S[(size_t)r * n + r];
  }
  return 0;
}

void orc_point_update(const orc_problem* p, int dA, int dC, const double* Vinv, const double* W,
                      const double* Y, const double* gb, const double* da, const double* dc,
                      double* db)
{
  int M = p->n_points;
  double* acc = (double*)malloc(sizeof(double) * 3 * (M > 0 ? M : 1));
  for (int j = 0; j < M; ++j) {
    for (int l = 0; l < 3; ++l) {
      double s = gb[3 * j + l];
      for (int c = 0; c < dC; ++c)
        if (c >= p->nnC) s -= Y[(size_t)j * 3 * dC + l * dC + c] * dc[c];
      acc[3 * j + l] = s;
    }
  }
  for (int k = 0; k < p->n_obs; ++k) {
    int i = p->view[k], j = p->point[k];
    if (i < p->nnA || j < p->nnB) continue;
    const double* Wk = W + (size_t)k * dA * 3;
    for (int l = 0; l < 3; ++l) {
      double s = 0.0;
      for (int r = 0; r < dA; ++r) s += Wk[r * 3 + l] * da[i * dA + r];
      acc[3 * j + l] -= s;
    }
  }
  for (int j = 0; j < M; ++j) {
    if (j < p->nnB) { db[3 * j] = db[3 * j + 1] = db[3 * j + 2] = 0.0; continue; }
    matmul(Vinv + 9 * (size_t)j, acc + 3 * j, db + 3 * j, 3, 3, 1);
  }
  free(acc);
}

void orc_rodrigues(const double omega[3], double R[9])
{
  /* createRotationMatrixRodrigues, V3D/include/Math/v3d_mathutilities.h:162-183 */
  double th = sqrt(omega[0] * omega[0] + omega[1] * omega[1] + omega[2] * omega[2]);
  memset(R, 0, 9 * sizeof(double));
  R[0] = R[4] = R[8] = 1.0;
  if (fabs(th) > 1e-6) {
    double J[9] = { 0.0, -omega[2], omega[1], omega[2], 0.0, -omega[0], -omega[1], omega[0], 0.0 };
    double J2[9];
    matmul(J, J, J2, 3, 3, 3);
    double c1 = sin(th) / th, c2 = (1.0 - cos(th)) / (th * th);
    for (int t = 0; t < 9; ++t) R[t] += c1 * J[t] + c2 * J2[t];
  }
}

static void update_intrinsics(int mode, const double* d, double* K, double* dist, double ar_fixed)
{
  /* mode fall-through of CommonInternals::updateParametersC (v3d_metricbundle.cpp:180-212) and
   * VaryingInternals::updateParametersA (:326-355).  d = [f, cx, cy, k1, k2, p1, p2]. ar_fixed < 0
   * means: use the current aspect ratio (VARYING). */
  int nint = intrinsic_dim(mode);
  if (nint >= 7) { dist[2] += d[5]; dist[3] += d[6]; }
  if (nint >= 5) { dist[0] += d[3]; dist[1] += d[4]; }
  if (nint >= 3) { K[2] += d[1]; K[5] += d[2]; }
  if (nint >= 1) {
    double ar = ar_fixed >= 0.0 ? ar_fixed : K[4] / K[0];
    K[0] += d[0];
    K[4] = ar * K[0];
  }
}

void orc_apply_update(const orc_problem* p, orc_params* x, double cached_ar,
                      const double* da, const double* db, const double* dc)
{
  int dA, dC;
  orc_dims(p->model, p->mode, &dA, &dC);
  for (int i = p->nnA; i < p->n_cams; ++i) {
    const double* d = da + (size_t)i * dA;
    double* T = x->T + 3 * i;
    double* R = x->R + 9 * i;
    T[0] += d[0]; T[1] += d[1]; T[2] += d[2];
    double dR[9], R0[9];
    orc_rodrigues(d + 3, dR);
    memcpy(R0, R, sizeof(R0));
    matmul(dR, R0, R, 3, 3, 3);
    if (p->model == ORC_MODEL_VARYING) update_intrinsics(p->mode, d + 6, x->K + 9 * i, x->dist + 4 * i, -1.0);
  }
  for (int j = p->nnB; j < p->n_points; ++j) {
    x->X[3 * j] += db[3 * j]; x->X[3 * j + 1] += db[3 * j + 1]; x->X[3 * j + 2] += db[3 * j + 2];
  }
  if (p->model == ORC_MODEL_COMMON && dC > p->nnC) update_intrinsics(p->mode, dc, x->K, x->dist, cached_ar);
}

static void copy_params(const orc_problem* p, const orc_params* s, orc_params* d)
{
  int N = p->n_cams, M = p->n_points;
  int nK = p->model == ORC_MODEL_STEREO ? 0 : (p->model == ORC_MODEL_COMMON ? 9 : 9 * N);
  int nD = p->model == ORC_MODEL_COMMON ? 4 : (p->model == ORC_MODEL_VARYING ? 4 * N : 0);
  if (nK) memcpy(d->K, s->K, sizeof(double) * nK);
  memcpy(d->R, s->R, sizeof(double) * 9 * N);
  memcpy(d->T, s->T, sizeof(double) * 3 * N);
  if (nD) memcpy(d->dist, s->dist, sizeof(double) * nD);
  memcpy(d->X, s->X, sizeof(double) * 3 * M);
}

/* SparseLevenbergOptimizer::minimize, v3d_optimization.cpp:719-1250, with the lambda schedule of
 * LevenbergOptimizerCommon (v3d_optimization.h:38-59). */
int orc_minimize(const orc_problem* p, orc_params* x, orc_options* opt, orc_result* res,
                 int* trace_iter, double* trace_lambda, double* trace_err, int trace_cap)
{
  int dA, dC;
  if (orc_dims(p->model, p->mode, &dA, &dC)) return -1;
  int N = p->n_cams, M = p->n_points, K = p->n_obs;
  int n = N * dA + dC;
  memset(res, 0, sizeof(*res));
  res->status = ORC_TIMEOUT;

  int nvA = N - p->nnA, nvB = M - p->nnB, nvC = dC - p->nnC;
  if (nvA <= 0 && nvB <= 0 && nvC <= 0) { res->status = ORC_CONVERGED; return 0; }

  double *w = malloc(sizeof(double) * (K ? K : 1)), *U = malloc(sizeof(double) * N * dA * dA + 8);
  double *V = malloc(sizeof(double) * 9 * M + 8), *W = malloc(sizeof(double) * (size_t)K * dA * 3 + 8);
  double *Xc = malloc(sizeof(double) * N * dA * (dC ? dC : 1)), *Y = malloc(sizeof(double) * 3 * M * (dC ? dC : 1));
  double *Z = malloc(sizeof(double) * 49), *ga = malloc(sizeof(double) * N * dA + 8);
  double *gb = malloc(sizeof(double) * 3 * M + 8), *gc = malloc(sizeof(double) * 8);
  double *S = malloc(sizeof(double) * (size_t)n * n + 8), *rhs = malloc(sizeof(double) * n + 8);
  double *Vinv = malloc(sizeof(double) * 9 * M + 8), *db = malloc(sizeof(double) * 3 * M + 8);
  int nK = p->model == ORC_MODEL_STEREO ? 0 : (p->model == ORC_MODEL_COMMON ? 9 : 9 * N);
  int nD = p->model == ORC_MODEL_COMMON ? 4 : (p->model == ORC_MODEL_VARYING ? 4 * N : 0);
  orc_params saved = { malloc(sizeof(double) * nK), malloc(sizeof(double) * 9 * N + 8),
                       malloc(sizeof(double) * 3 * N + 8), malloc(sizeof(double) * (nD ? nD : 1)),
                       malloc(sizeof(double) * 3 * M + 8) };

  int compute_derivatives = 1, it;
  double err = 0.0;
  double lambda = opt->lambda;
  for (it = 0; it < opt->max_iterations; ++it) {
    if (compute_derivatives) {
      err = orc_normal_blocks(p, x, opt->cached_aspect_ratio, w, U, V, W, Xc, Y, Z, ga, gb, gc);
      res->n_relinearizations++;
      res->final_err = err;
      if (trace_cap > 0 && res->n_relinearizations <= trace_cap) {
        int t = res->n_relinearizations - 1;
        trace_iter[t] = it; trace_lambda[t] = lambda; trace_err[t] = err;
      }
      /* gradient stopping criterion, cpp:857-861 */
      double gmax = 0.0;
      for (int t = 0; t < N * dA; ++t) gmax = fmax(gmax, fabs(ga[t]));
      for (int t = 0; t < 3 * M; ++t) gmax = fmax(gmax, fabs(gb[t]));
      for (int t = p->nnC; t < dC; ++t) gmax = fmax(gmax, fabs(gc[t]));
      if (gmax < opt->gradient_threshold) { res->status = ORC_CONVERGED; break; }
      if (it == 0) {
        /* initial lambda = tau * max diagonal, cpp:981-1052 */
        double m = -1e30;
        for (int i = p->nnA; i < N; ++i)
          for (int l = 0; l < dA; ++l) m = fmax(m, U[(size_t)i * dA * dA + l * dA + l]);
        for (int j = p->nnB; j < M; ++j)
          for (int l = 0; l < 3; ++l) m = fmax(m, V[9 * (size_t)j + 4 * l]);
        for (int l = p->nnC; l < dC; ++l) m = fmax(m, Z[l * dC + l]);
        lambda = opt->tau * m;
      }
    }

    int success = !orc_reduced_system(p, dA, dC, lambda, U, V, W, Xc, Y, Z, ga, gb, gc, S, rhs, Vinv);
    if (success) success = !orc_cholesky_solve(n, S, rhs);
    double rho = 0.0;
    if (success) {
      const double* da = rhs;
      const double* dc = rhs + N * dA;
      orc_point_update(p, dA, dC, Vinv, W, Y, gb, da, dc, db);
      /* |delta|^2 and delta . J^T e over the varying parameters */
      double d2 = 0.0, dg = 0.0;
      for (int i = p->nnA; i < N; ++i)
        for (int l = 0; l < dA; ++l) { double v = da[i * dA + l]; d2 += v * v; dg += v * ga[i * dA + l]; }
      for (int j = p->nnB; j < M; ++j)
        for (int l = 0; l < 3; ++l) { double v = db[3 * j + l]; d2 += v * v; dg += v * gb[3 * j + l]; }
      for (int l = p->nnC; l < dC; ++l) { d2 += dc[l] * dc[l]; dg += dc[l] * gc[l]; }
      /* update stopping criterion, cpp:1154-1159 */
      if (sqrt(d2) < opt->update_threshold * (opt->param_length + opt->update_threshold)) {
        res->status = ORC_SMALL_UPDATE;
        break;
      }
      copy_params(p, x, &saved);
      orc_apply_update(p, x, opt->cached_aspect_ratio, da, db, dc);
      double new_err = orc_cost(p, x, opt->cached_aspect_ratio, w);   /* Q2: old weights */
      rho = (err - new_err) / (lambda * d2 + dg);
    }
    if (success && rho > 0.0) {
      double r = 2.0 * rho - 1.0;
      double f = 1.0 - r * r * r;
      lambda *= (f > 1.0 / 3.0 ? f : 1.0 / 3.0);
      if (lambda < 1e-10) lambda = 1e-10;
      opt->nu = 2.0;
      compute_derivatives = 1;
    } else {
      if (success) copy_params(p, &saved, x);
      res->n_rejected++;
      lambda *= opt->nu;
      opt->nu *= 2.0;
      compute_derivatives = 0;
    }
  }
  res->iterations = it;
  opt->lambda = lambda;

  free(w); free(U); free(V); free(W); free(Xc); free(Y); free(Z); free(ga); free(gb); free(gc);
  free(S); free(rhs); free(Vinv); free(db);
  free(saved.K); free(saved.R); free(saved.T); free(saved.dist); free(saved.X);
  return 0;
}

int orc_pcg(int n, int bs, const double* S, const double* b, const double* Minv, double rel_tol,
            int max_iter, double* x)
{
  int nb = n / bs;
  double* Mi = NULL;
  if (!Minv) {
    /* block-Jacobi: invert each diagonal block by Gauss-Jordan */
    Mi = (double*)malloc(sizeof(double) * nb * bs * bs);
    double* a = (double*)malloc(sizeof(double) * bs * 2 * bs);
    for (int q = 0; q < nb; ++q) {
      for (int r = 0; r < bs; ++r)
        for (int c = 0; c < 2 * bs; ++c)
          a[r * 2 * bs + c] = c < bs ? S[(size_t)(q * bs + r) * n + q * bs + c] : (c - bs == r ? 1.0 : 0.0);
      for (int c = 0; c < bs; ++c) {
        double piv = a[c * 2 * bs + c];
        for (int t = 0; t < 2 * bs; ++t) a[c * 2 * bs + t] /= piv;
        for (int r = 0; r < bs; ++r) {
          if (r == c) continue;
          double f = a[r * 2 * bs + c];
          for (int t = 0; t < 2 * bs; ++t) a[r * 2 * bs + t] -= f * a[c * 2 * bs + t];
        }
      }
      for (int r = 0; r < bs; ++r)
        for (int c = 0; c < bs; ++c) Mi[(size_t)q * bs * bs + r * bs + c] = a[r * 2 * bs + bs + c];
    }
    free(a);
    Minv = Mi;
  }
  double *r = malloc(sizeof(double) * n), *z = malloc(sizeof(double) * n);
  double *pp = malloc(sizeof(double) * n), *Ap = malloc(sizeof(double) * n);
  double bnorm = 0.0;
  for (int t = 0; t < n; ++t) { x[t] = 0.0; r[t] = b[t]; bnorm += b[t] * b[t]; }
  bnorm = sqrt(bnorm);
  int it = 0;
  double rz = 0.0;
  for (int q = 0; q < nb; ++q) matmul(Minv + (size_t)q * bs * bs, r + q * bs, z + q * bs, bs, bs, 1);
  for (int t = 0; t < n; ++t) { pp[t] = z[t]; rz += r[t] * z[t]; }
  if (bnorm == 0.0) goto done;
  for (it = 0; it < max_iter; ++it) {
    double rn = 0.0;
    for (int t = 0; t < n; ++t) rn += r[t] * r[t];
    if (sqrt(rn) <= rel_tol * bnorm) break;
    double pAp = 0.0;
    for (int rr = 0; rr < n; ++rr) {
      double s = 0.0;
      for (int c = 0; c < n; ++c) s += S[(size_t)rr * n + c] * pp[c];
      Ap[rr] = s;
      pAp += pp[rr] * s;
    }
    double alpha = rz / pAp;
    for (int t = 0; t < n; ++t) { x[t] += alpha * pp[t]; r[t] -= alpha * Ap[t]; }
    for (int q = 0; q < nb; ++q) matmul(Minv + (size_t)q * bs * bs, r + q * bs, z + q * bs, bs, bs, 1);
    double rz_new = 0.0;
    for (int t = 0; t < n; ++t) rz_new += r[t] * z[t];
    double beta = rz_new / rz;
    rz = rz_new;
    for (int t = 0; t < n; ++t) pp[t] = z[t] + beta * pp[t];
  }
done:
  free(r); free(z); free(pp); free(Ap);
  if (Mi) free(Mi);
  return it;
}

/* ---- Rotation averaging (SparseRotationOptimizer, v3d_mviewutilities.cpp:470-582) ---------- */

/* e = R_j - R_ij R_i (evalResidual, v3d_mviewutilities.cpp:486-508). */
static void rot_residual(const double* Ri, const double* Rj, const double* Rij, double* e)
{
  double P[9];
  matmul(Rij, Ri, P, 3, 3, 3);
  for (int t = 0; t < 9; ++t) e[t] = Rj[t] - P[t];
}

/* 9x3 Jacobian of vec(A (I + [w]x)) at w = 0 (fillJacobians, :510-553): A = -R_ij R_i for the
 * first view of the pair, R_j for the second. */
static void rot_jacobian(const double* A, double* J)
{
  for (int r = 0; r < 3; ++r) {
    const double* a = A + 3 * r;
    double* j0 = J + 9 * r;          /* rows 3r, 3r+1, 3r+2 of the 9x3 matrix */
    j0[0] = 0.0;   j0[1] = -a[2]; j0[2] = a[1];
    j0[3] = a[2];  j0[4] = 0.0;   j0[5] = -a[0];
    j0[6] = -a[1]; j0[7] = a[0];  j0[8] = 0.0;
  }
}

double orc_rotations_cost(int n_views, int n_pairs, const double* rel, const int* pairs, const double* R)
{
  (void)n_views;
  double err = 0.0, e[9];
  for (int k = 0; k < 2 * n_pairs; ++k) {
    int q = k < n_pairs ? k : k - n_pairs;
    rot_residual(R + 9 * pairs[2 * q], R + 9 * pairs[2 * q + 1], rel + 9 * q, e);
    for (int t = 0; t < 9; ++t) err += e[t] * e[t];
  }
  return err;
}

/* Solve (U + lambda I) d = g for one 3x3 block by the up-looking LDL^T of LDL_numeric /
 * LDL_lsolve / LDL_dsolve / LDL_ltsolve (v3d_optimization.cpp:102-230) in natural order.
 * Returns 1 when a pivot D(k,k) is exactly zero (the reference then rejects the step). */
static int rot_ldl_solve(const double* U, double lambda, const double* g, double* d)
{
  double a00 = U[0] + lambda, a11 = U[4] + lambda, a22 = U[8] + lambda;
  double a01 = U[1], a02 = U[2], a12 = U[5];
  double D0 = a00;
  if (D0 == 0.0) return 1;
  double L10 = a01 / D0;
  double D1 = a11 - L10 * a01;
  if (D1 == 0.0) return 1;
  double y1 = a12 - L10 * a02;          /* Y[1] -= L10 * y0 while processing column 0 of row 2 */
  double L20 = a02 / D0;
  double D2 = a22 - L20 * a02;
  double L21 = y1 / D1;
  D2 -= L21 * y1;
  if (D2 == 0.0) return 1;
  double x0 = g[0], x1 = g[1], x2 = g[2];
  x1 -= L10 * x0; x2 -= L20 * x0; x2 -= L21 * x1;
  x0 /= D0; x1 /= D1; x2 /= D2;
  x1 -= L21 * x2; x0 -= L10 * x1; x0 -= L20 * x2;
  d[0] = x0; d[1] = x1; d[2] = x2;
  return 0;
}

int orc_rotations_minimize(int n_views, int n_pairs, const double* rel, const int* pairs, double* R,
                           orc_options* opt, orc_result* res, double* trace_err, int trace_cap)
{
  int N = n_views, P = n_pairs, K = 2 * n_pairs;
  memset(res, 0, sizeof(*res));
  res->status = ORC_TIMEOUT;
  if (N <= 0) { res->status = ORC_CONVERGED; return 0; }
  double *U = calloc((size_t)9 * N, sizeof(double)), *g = calloc((size_t)3 * N, sizeof(double));
  double *d = calloc((size_t)3 * N, sizeof(double)), *Rs = malloc(sizeof(double) * 9 * N);
  double plen = sqrt(3.0 * N);
  int compute_derivatives = 1, it;
  double err = 0.0, lambda = opt->lambda;
  for (it = 0; it < opt->max_iterations; ++it) {
    if (compute_derivatives) {
      memset(U, 0, sizeof(double) * 9 * N);
      memset(g, 0, sizeof(double) * 3 * N);
      err = 0.0;
      double e[9], J[27], A[9];
      for (int k = 0; k < K; ++k) {
        int q = k < P ? k : k - P;
        const double *Ri = R + 9 * pairs[2 * q], *Rj = R + 9 * pairs[2 * q + 1], *Rij = rel + 9 * q;
        rot_residual(Ri, Rj, Rij, e);
        for (int t = 0; t < 9; ++t) err += e[t] * e[t];
      }
      for (int k = 0; k < K; ++k) {
        int q = k < P ? k : k - P;
        int view = k < P ? pairs[2 * q] : pairs[2 * q + 1];
        const double *Ri = R + 9 * pairs[2 * q], *Rj = R + 9 * pairs[2 * q + 1], *Rij = rel + 9 * q;
        rot_residual(Ri, Rj, Rij, e);
        if (k < P) { matmul(Rij, Ri, A, 3, 3, 3); for (int t = 0; t < 9; ++t) A[t] = -A[t]; }
        else memcpy(A, Rj, sizeof(A));
        rot_jacobian(A, J);
        double* Uv = U + 9 * (size_t)view;
        double* gv = g + 3 * (size_t)view;
        for (int a = 0; a < 3; ++a) {
          double s = 0.0;
          for (int r = 0; r < 9; ++r) s += J[3 * r + a] * -e[r];
          gv[a] += s;
          for (int b = 0; b < 3; ++b) {
            double u = 0.0;
            for (int r = 0; r < 9; ++r) u += J[3 * r + a] * J[3 * r + b];
            Uv[3 * a + b] += u;
          }
        }
      }
      res->n_relinearizations++;
      res->final_err = err;
      if (trace_cap > 0 && res->n_relinearizations <= trace_cap) trace_err[res->n_relinearizations - 1] = err;
      double gmax = 0.0;
      for (int t = 0; t < 3 * N; ++t) gmax = fmax(gmax, fabs(g[t]));
      if (gmax < opt->gradient_threshold) { res->status = ORC_CONVERGED; break; }
      if (it == 0) {
        double m = -1e30;
        for (int i = 0; i < N; ++i)
          for (int l = 0; l < 3; ++l) m = fmax(m, U[9 * (size_t)i + 4 * l]);
        lambda = opt->tau * m;
      }
    }
    int success = 1;
    for (int i = 0; i < N && success; ++i)
      if (rot_ldl_solve(U + 9 * (size_t)i, lambda, g + 3 * (size_t)i, d + 3 * (size_t)i)) success = 0;
    double rho = 0.0;
    if (success) {
      double d2 = 0.0, dg = 0.0;
      for (int t = 0; t < 3 * N; ++t) d2 += d[t] * d[t];
      if (sqrt(d2) < opt->update_threshold * (plen + opt->update_threshold)) {
        res->status = ORC_SMALL_UPDATE;
        break;
      }
      memcpy(Rs, R, sizeof(double) * 9 * N);
      for (int i = 0; i < N; ++i) {
        double dR[9];
        orc_rodrigues(d + 3 * i, dR);
        matmul(Rs + 9 * i, dR, R + 9 * i, 3, 3, 3);
      }
      double new_err = orc_rotations_cost(N, P, rel, pairs, R);
      for (int t = 0; t < 3 * N; ++t) dg += d[t] * g[t];
      rho = (err - new_err) / (lambda * d2 + dg);
    }
    if (success && rho > 0.0) {
      double r = 2.0 * rho - 1.0;
      double f = 1.0 - r * r * r;
      lambda *= (f > 1.0 / 3.0 ? f : 1.0 / 3.0);
      if (lambda < 1e-10) lambda = 1e-10;
      opt->nu = 2.0;
      compute_derivatives = 1;
    } else {
      if (success) memcpy(R, Rs, sizeof(double) * 9 * N);
      res->n_rejected++;
      lambda *= opt->nu;
      opt->nu *= 2.0;
      compute_derivatives = 0;
    }
  }
  res->iterations = it;
  opt->lambda = lambda;
  free(U); free(g); free(d); free(Rs);
  return 0;
}

