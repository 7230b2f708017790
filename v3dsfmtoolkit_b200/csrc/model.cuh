// Per-observation camera models of the metric bundle adjuster, FP64 device code.
//
// Projection and analytic Jacobians of the three reference models:
//   STD     : StdMetricBundleOptimizer (V3D/include/Geometry/v3d_metricbundle.h:121-132,
//             V3D/src/Geometry/v3d_metricbundle.cpp:52-98; CameraMatrix::projectPoint,
//             V3D/include/Geometry/v3d_cameramatrix.h:184-190)
//   COMMON  : CommonInternalsMetricBundleOptimizer (v3d_metricbundle.h:185-209,
//             v3d_metricbundle.cpp:102-178)
//   VARYING : VaryingInternalsMetricBundleOptimizer (v3d_metricbundle.h:275-291,
//             v3d_metricbundle.cpp:216-296)
//   STEREO  : StereoMetricBundleOptimizer (V3D/include/Geometry/v3d_stereobundle.h:66-80,
//             V3D/src/Geometry/v3d_stereobundle.cpp:11-67): the rig pose (R, T) moves the point
//             into rig space, rig camera l (K_l, R_l, T_l) projects it like STD; the Jacobian
//             is the STD one of camera l composed with R_l (f and aspect ratio of K_l).
// with the Brown distortion of V3D/include/Geometry/v3d_distortion.h:18-72.
//
// The Jacobian is d e / d p for e = proj - m.  Camera columns are (T, omega) first, then for
// VARYING the intrinsic columns [f, cx, cy, k1, k2, p1, p2] up to the mode's count.  COMMON
// puts those intrinsic columns into the global block C instead.  Reference behaviours kept:
// the STD Jacobian ignores skew and principal point; d/df uses the distorted point on both
// rows; FULL_BUNDLE_NO_ROTATIONS zeroes the translation columns (the first three).
#pragma once

#include "common.cuh"

namespace v3dba {

enum { kModelStd = 0, kModelCommon = 1, kModelVarying = 2, kModelStereo = 3 };

__host__ __device__ constexpr int intrinsic_dim(int mode) {
  return mode == 1 ? 1 : mode == 2 ? 3 : mode == 3 ? 5 : mode == 4 ? 7 : 0;
}

// Camera parameters gathered for one observation.
struct Cam {
  double R[9], T[3];
  double K[9];                      // intrinsics, row-major (STD uses all of K; STEREO: K_l)
  double d[4];                      // k1 k2 p1 p2
  double Rl[9], Tl[3];              // STEREO: pose of the rig camera on the rig
};

template <int MODEL>
__device__ __forceinline__ void load_cam(Cam& c, const double* __restrict__ R, const double* __restrict__ T,
                                         const double* __restrict__ K, const double* __restrict__ dist,
                                         int i) {
#pragma unroll
  for (int t = 0; t < 9; ++t) c.R[t] = __ldg(R + 9 * i + t);
#pragma unroll
  for (int t = 0; t < 3; ++t) c.T[t] = __ldg(T + 3 * i + t);
  if (MODEL != kModelStereo) {   // STEREO takes K from the rig camera (load_rig)
    const double* k = (MODEL == kModelCommon) ? K : K + 9 * i;
#pragma unroll
    for (int t = 0; t < 9; ++t) c.K[t] = __ldg(k + t);
  }
  if (MODEL == kModelCommon || MODEL == kModelVarying) {
    const double* dd = (MODEL == kModelCommon) ? dist : dist + 4 * i;
#pragma unroll
    for (int t = 0; t < 4; ++t) c.d[t] = __ldg(dd + t);
  } else {
    c.d[0] = c.d[1] = c.d[2] = c.d[3] = 0.0;
  }
}

// Rig camera l of a STEREO observation: K_l, R_l, T_l from rig[l * 24 ...] (K 9, R 9, T 3).
__device__ __forceinline__ void load_rig(Cam& c, const double* __restrict__ rig, int l) {
  const double* r = rig + 24 * (size_t)l;
#pragma unroll
  for (int t = 0; t < 9; ++t) c.K[t] = __ldg(r + t);
#pragma unroll
  for (int t = 0; t < 9; ++t) c.Rl[t] = __ldg(r + 9 + t);
#pragma unroll
  for (int t = 0; t < 3; ++t) c.Tl[t] = __ldg(r + 18 + t);
}

// e = proj(X) - m.  Returns the camera-space point in XX.
template <int MODEL>
__device__ __forceinline__ void residual(const Cam& c, const double X[3], double mx, double my,
                                         double XX[3], double e[2]) {
#pragma unroll
  for (int r = 0; r < 3; ++r) XX[r] = c.R[3 * r] * X[0] + c.R[3 * r + 1] * X[1] + c.R[3 * r + 2] * X[2] + c.T[r];
  if (MODEL == kModelStereo) {   // into the rig camera: R_l Y + T_l
    double Y[3] = {XX[0], XX[1], XX[2]};
#pragma unroll
    for (int r = 0; r < 3; ++r) XX[r] = c.Rl[3 * r] * Y[0] + c.Rl[3 * r + 1] * Y[1] + c.Rl[3 * r + 2] * Y[2] + c.Tl[r];
  }
  if (MODEL == kModelStd || MODEL == kModelStereo) {
    // K (R X + T) dehomogenised, with the full 3x3 K
    const double h0 = c.K[0] * XX[0] + c.K[1] * XX[1] + c.K[2] * XX[2];
    const double h1 = c.K[3] * XX[0] + c.K[4] * XX[1] + c.K[5] * XX[2];
    const double h2 = c.K[6] * XX[0] + c.K[7] * XX[1] + c.K[8] * XX[2];
    e[0] = h0 / h2 - mx;
    e[1] = h1 / h2 - my;
  } else {
    const double ux = XX[0] / XX[2], uy = XX[1] / XX[2];
    const double r2 = ux * ux + uy * uy;
    const double kr = 1.0 + c.d[0] * r2 + c.d[1] * r2 * r2;
    const double xd = kr * ux + 2.0 * c.d[2] * ux * uy + c.d[3] * (r2 + 2.0 * ux * ux);
    const double yd = kr * uy + 2.0 * c.d[3] * ux * uy + c.d[2] * (r2 + 2.0 * uy * uy);
    e[0] = c.K[0] * xd + c.K[1] * yd + c.K[2] - mx;
    e[1] = c.K[4] * yd + c.K[5] - my;
  }
}

// Residual and raw Jacobian blocks of one observation.
//   A : 2 x DA (camera), B : 2 x 3 (point), C : 2 x DC (global intrinsics, COMMON only).
template <int MODEL, int DA, int DC>
__device__ __forceinline__ void linearize_obs(const Cam& c, const double X[3], double mx, double my,
                                              int mode, double cached_ar, double e[2],
                                              double A[2][DA], double B[2][3], double (&C)[2][DC > 0 ? DC : 1]) {
  double XX[3];
  residual<MODEL>(c, X, mx, my, XX, e);

  // d XX / d (T, omega) = [ I | -[R X]_x ],  d XX / d X = R  (R X recovered as XX - T); STEREO
  // composes both with R_l (the pose moves the point in rig space)
  double v0, v1, v2;
  if (MODEL == kModelStereo) {
    v0 = c.R[0] * X[0] + c.R[1] * X[1] + c.R[2] * X[2];
    v1 = c.R[3] * X[0] + c.R[4] * X[1] + c.R[5] * X[2];
    v2 = c.R[6] * X[0] + c.R[7] * X[1] + c.R[8] * X[2];
  } else {
    v0 = XX[0] - c.T[0]; v1 = XX[1] - c.T[1]; v2 = XX[2] - c.T[2];
  }
  const double iz = 1.0 / XX[2];

  double P[2][3];  // d proj / d XX (STEREO: d proj / d Y = d proj / d XX * R_l)
  double fx, fy, ux = 0.0, uy = 0.0, xd = 0.0, yd = 0.0;
  if (MODEL == kModelStd || MODEL == kModelStereo) {
    const double f = c.K[0], ar = c.K[4] / c.K[0];
    const double bx = f / (XX[2] * XX[2]), by = ar * bx;
    P[0][0] = bx * XX[2]; P[0][1] = 0.0;        P[0][2] = -bx * XX[0];
    P[1][0] = 0.0;        P[1][1] = by * XX[2]; P[1][2] = -by * XX[1];
    fx = f; fy = ar * f;
    if (MODEL == kModelStereo) {
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const double p0 = P[r][0], p1 = P[r][1], p2 = P[r][2];
#pragma unroll
        for (int q = 0; q < 3; ++q) P[r][q] = p0 * c.Rl[q] + p1 * c.Rl[3 + q] + p2 * c.Rl[6 + q];
      }
    }
  } else {
    const double f = c.K[0];
    const double ar = (MODEL == kModelCommon) ? cached_ar : c.K[4] / c.K[0];
    fx = f; fy = ar * f;
    ux = XX[0] * iz; uy = XX[1] * iz;
    const double r2 = ux * ux + uy * uy;
    const double kr = 1.0 + c.d[0] * r2 + c.d[1] * r2 * r2;
    const double dkr = 2.0 * c.d[0] + 4.0 * c.d[1] * r2;
    xd = kr * ux + 2.0 * c.d[2] * ux * uy + c.d[3] * (r2 + 2.0 * ux * ux);
    yd = kr * uy + 2.0 * c.d[3] * ux * uy + c.d[2] * (r2 + 2.0 * uy * uy);
    const double j00 = kr + ux * ux * dkr + 2.0 * c.d[2] * uy + 6.0 * c.d[3] * ux;
    const double j01 = ux * uy * dkr + 2.0 * c.d[2] * ux + 2.0 * c.d[3] * uy;
    const double j11 = kr + uy * uy * dkr + 6.0 * c.d[2] * uy + 2.0 * c.d[3] * ux;
    // d proj / d xu = diag(fx, fy) * J_dist;  d xu / d XX = [[1/z, 0, -x/z^2], [0, 1/z, -y/z^2]]
    const double a00 = fx * j00, a01 = fx * j01, a10 = fy * j01, a11 = fy * j11;
    const double iz2 = iz * iz;
    const double dx2 = -XX[0] * iz2, dy2 = -XX[1] * iz2;
    P[0][0] = a00 * iz; P[0][1] = a01 * iz; P[0][2] = a00 * dx2 + a01 * dy2;
    P[1][0] = a10 * iz; P[1][1] = a11 * iz; P[1][2] = a10 * dx2 + a11 * dy2;
  }

  const bool no_trans = (MODEL == kModelCommon || MODEL == kModelVarying) && (mode == -1);
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    // translation columns: P * I
    A[r][0] = no_trans ? 0.0 : P[r][0];
    A[r][1] = no_trans ? 0.0 : P[r][1];
    A[r][2] = no_trans ? 0.0 : P[r][2];
    // rotation columns: P * (-[v]_x) with -[v]_x = [[0, v2, -v1], [-v2, 0, v0], [v1, -v0, 0]]
    A[r][3] = -P[r][1] * v2 + P[r][2] * v1;
    A[r][4] = P[r][0] * v2 - P[r][2] * v0;
    A[r][5] = -P[r][0] * v1 + P[r][1] * v0;
#pragma unroll
    for (int q = 0; q < 3; ++q)
      B[r][q] = P[r][0] * c.R[q] + P[r][1] * c.R[3 + q] + P[r][2] * c.R[6 + q];
  }

  if (MODEL == kModelCommon || MODEL == kModelVarying) {
    const int nint = intrinsic_dim(mode);
    // intrinsic columns [f, cx, cy, k1, k2, p1, p2]
    double G[2][7];
    const double r2 = ux * ux + uy * uy;
    G[0][0] = xd; G[1][0] = yd;
    G[0][1] = 1.0; G[0][2] = 0.0; G[1][1] = 0.0; G[1][2] = 1.0;
    G[0][3] = fx * ux * r2; G[0][4] = fx * ux * r2 * r2;
    G[1][3] = fy * uy * r2; G[1][4] = fy * uy * r2 * r2;
    G[0][5] = fx * 2.0 * ux * uy; G[0][6] = fx * (r2 + 2.0 * ux * ux);
    G[1][5] = fy * (r2 + 2.0 * uy * uy); G[1][6] = fy * 2.0 * ux * uy;
    if (MODEL == kModelCommon) {
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int q = 0; q < (DC > 0 ? DC : 1); ++q) C[r][q] = (q < nint && DC > 0) ? G[r][q] : 0.0;
    } else {
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int q = 6; q < DA; ++q) A[r][q] = (q - 6 < nint) ? G[r][q - 6] : 0.0;
    }
  }
}

__device__ __forceinline__ double huber_weight(double thr, const double e[2]) {
  const double n = sqrt(e[0] * e[0] + e[1] * e[1]);
  return (n < thr) ? 1.0 : sqrt(thr / n);
}

// createRotationMatrixRodrigues (V3D/include/Math/v3d_mathutilities.h:162-183) followed by
// R <- dR * R (v3d_metricbundle.cpp:31-37).
__device__ __forceinline__ void rotate_update(const double w[3], double R[9]) {
  const double th = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  double dR[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (fabs(th) > 1e-6) {
    const double J[9] = {0.0, -w[2], w[1], w[2], 0.0, -w[0], -w[1], w[0], 0.0};
    double J2[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        J2[3 * r + q] = J[3 * r] * J[q] + J[3 * r + 1] * J[3 + q] + J[3 * r + 2] * J[6 + q];
    const double c1 = sin(th) / th, c2 = (1.0 - cos(th)) / (th * th);
#pragma unroll
    for (int t = 0; t < 9; ++t) dR[t] += c1 * J[t] + c2 * J2[t];
  }
  double R0[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) R0[t] = R[t];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int q = 0; q < 3; ++q)
      R[3 * r + q] = dR[3 * r] * R0[q] + dR[3 * r + 1] * R0[3 + q] + dR[3 * r + 2] * R0[6 + q];
}

// Intrinsic update of CommonInternals::updateParametersC (v3d_metricbundle.cpp:180-212) and
// VaryingInternals::updateParametersA (:326-355); d = [f, cx, cy, k1, k2, p1, p2].
// ar_fixed < 0: keep the current aspect ratio (VARYING); else K11 = ar_fixed * K00 (COMMON).
__host__ __device__ __forceinline__ void intrinsic_update(int mode, const double* d, double* K,
                                                          double* dist, double ar_fixed) {
  const int nint = intrinsic_dim(mode);
  if (nint >= 7) { dist[2] += d[5]; dist[3] += d[6]; }
  if (nint >= 5) { dist[0] += d[3]; dist[1] += d[4]; }
  if (nint >= 3) { K[2] += d[1]; K[5] += d[2]; }
  if (nint >= 1) {
    const double ar = ar_fixed >= 0.0 ? ar_fixed : K[4] / K[0];
    K[0] += d[0];
    K[4] = ar * K[0];
  }
}

}  // namespace v3dba
