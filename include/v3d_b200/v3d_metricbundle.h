// -*- C++ -*-
// Drop-in replacement of the reference header Geometry/v3d_metricbundle.h for the metric bundle
// adjusters, running on the B200 through the C-ABI of v3dba.h.
//
// A caller keeps its code and swaps
//     #include "Geometry/v3d_metricbundle.h"
// for
//     #include "v3d_b200/v3d_metricbundle.h"
// and links libv3dba.so.  The classes keep the reference's names, constructor signatures,
// public fields and minimize() (V3D/include/Geometry/v3d_metricbundle.h:16-320,
// V3D/include/Math/v3d_optimization.h:25-68, 272-407):
//
//   StdMetricBundleOptimizer(inlierThreshold, cams, Xs, measurements, view, point)
//   CommonInternalsMetricBundleOptimizer(mode, inlierThreshold, K, distortion, cams, Xs, ...)
//   VaryingInternalsMetricBundleOptimizer(mode, inlierThreshold, distortions, cams, Xs, ...)
//   StdDistortionMetricBundleOptimizer   (alias of CommonInternalsMetricBundleOptimizer)
//
// The optimizer holds references, as the reference does; minimize() updates the cameras,
// points, K and distortion(s) in place.  The reference's own headers for CameraMatrix,
// StdDistortionFunction, Vector/Matrix and LevenbergOptimizerCommon (status codes, tau,
// lambda, thresholds, optimizerVerbosenessLevel) are used unchanged.
//
// Differences, all deliberate:
//   * maxIterations defaults to 50 (LevenbergOptimizerCommon's value): the reference's
//     SparseLevenbergOptimizer redeclares it uninitialised (v3d_optimization.h:382); every
//     reference caller sets it.
//   * Fixed parameters (setNonvaryingCounts) are handled exactly; the reference mixes
//     observations of fixed cameras into W_0 (v3d_optimization.cpp:313, 930).
//   * Errors of the GPU path (CUDA failure, invalid input) are reported on stderr, kept in
//     lastError, and leave status = LEVENBERG_OPTIMIZER_TIMEOUT with the parameters untouched
//     (the reference has no error path other than the status).
//   * `precision` selects the arithmetic of the normal-equation blocks (V3DBA_PRECISION_MIXED by
//     default, V3DBA_PRECISION_FP64).
#ifndef V3D_B200_METRICBUNDLE_H
#define V3D_B200_METRICBUNDLE_H

#include <cmath>
#include <cstdio>
#include <vector>

#include "Geometry/v3d_cameramatrix.h"
#include "Geometry/v3d_distortion.h"
#include "Math/v3d_linear.h"
#include "Math/v3d_optimization.h"

#include "v3dba.h"

namespace V3D
{
   using std::vector;

   // The C-ABI reads measurements and points in place from the caller's vectors.
   static_assert(sizeof(Vector2d) == 2 * sizeof(double), "Vector2d must be two packed doubles");
   static_assert(sizeof(Vector3d) == 3 * sizeof(double), "Vector3d must be three packed doubles");

   enum
   {
      FULL_BUNDLE_NO_ROTATIONS = V3DBA_FULL_BUNDLE_NO_ROTATIONS,
      FULL_BUNDLE_METRIC = V3DBA_FULL_BUNDLE_METRIC,
      FULL_BUNDLE_FOCAL_LENGTH = V3DBA_FULL_BUNDLE_FOCAL_LENGTH,
      FULL_BUNDLE_FOCAL_LENGTH_PP = V3DBA_FULL_BUNDLE_FOCAL_LENGTH_PP,
      FULL_BUNDLE_RADIAL = V3DBA_FULL_BUNDLE_RADIAL,
      FULL_BUNDLE_RADIAL_TANGENTIAL = V3DBA_FULL_BUNDLE_RADIAL_TANGENTIAL
   };

   //! Common part of the three metric bundle adjusters: packs the caller's cameras and points
   //! into the structure-of-arrays layout of the C-ABI, runs v3dba_minimize, writes back.
   struct MetricBundleOptimizerBase : public LevenbergOptimizerCommon
   {
         MetricBundleOptimizerBase(int model, int mode, double inlierThreshold,
                                   vector<CameraMatrix>& cams, vector<Vector3d>& Xs,
                                   vector<Vector2d> const& measurements,
                                   vector<int> const& corrspondingView,
                                   vector<int> const& corrspondingPoint,
                                   Matrix3x3d* K, StdDistortionFunction* distortion,
                                   vector<StdDistortionFunction>* distortions)
            : LevenbergOptimizerCommon(),
              precision(V3DBA_PRECISION_MIXED), lastError(V3DBA_OK),
              _model(model), _mode(mode), _cams(cams), _Xs(Xs), _K(K), _distortion(distortion),
              _distortions(distortions), _handle(0), _nnA(0), _nnB(0), _nnC(0)
         {
            int const N = cams.size(), M = Xs.size(), Kn = measurements.size();
            std::vector<double> Kb, R, T, D;
            pack(Kb, R, T, D);
            v3dba_problem p = v3dba_problem();
            p.model = model; p.mode = mode;
            p.n_cameras = N; p.n_points = M; p.n_measurements = Kn;
            p.inlier_threshold = inlierThreshold;
            p.K = Kb.data(); p.R = R.data(); p.T = T.data();
            p.dist = D.empty() ? 0 : D.data(); p.X = points();
            // the measurements are passed in place: a vector<Vector2d> is 2 doubles per element
            p.measurements = Kn ? measurements[0].begin() : 0;
            p.view = corrspondingView.data(); p.point = corrspondingPoint.data();
            lastError = v3dba_create(&p, &_handle);
            if (lastError != V3DBA_OK)
            {
               std::fprintf(stderr, "v3dba_create failed: %s\n", v3dba_error_string(lastError));
               _handle = 0;
            }
         }

         virtual ~MetricBundleOptimizerBase() { if (_handle) v3dba_destroy(_handle); }

         void setNonvaryingCounts(int nNonvaryingA, int nNonvaryingB, int nNonvaryingC)
         {
            _nnA = nNonvaryingA; _nnB = nNonvaryingB; _nnC = nNonvaryingC;
         }

         void getNonvaryingCounts(int& nNonvaryingA, int& nNonvaryingB, int& nNonvaryingC) const
         {
            nNonvaryingA = _nnA; nNonvaryingB = _nnB; nNonvaryingC = _nnC;
         }

         void minimize()
         {
            status = LEVENBERG_OPTIMIZER_TIMEOUT;
            if (!_handle) return;
            std::vector<double> Kb, R, T, D;
            pack(Kb, R, T, D);
            int rc = v3dba_set_params(_handle, Kb.data(), R.data(), T.data(), D.empty() ? 0 : D.data(), points());
            if (rc == V3DBA_OK) rc = v3dba_set_nonvarying(_handle, _nnA, _nnB, _nnC);
            if (rc == V3DBA_OK) rc = v3dba_set_lambda(_handle, lambda);
            v3dba_options o;
            v3dba_default_options(&o);
            o.tau = tau; o.max_iterations = maxIterations;
            o.gradient_threshold = gradientThreshold; o.update_threshold = updateThreshold;
            o.verbosity = optimizerVerbosenessLevel;
            o.precision = precision;
            v3dba_result r;
            if (rc == V3DBA_OK) rc = v3dba_minimize(_handle, &o, &r);
            if (rc == V3DBA_OK) rc = v3dba_get_params(_handle, Kb.data(), R.data(), T.data(), D.empty() ? 0 : D.data(), points());
            lastError = rc;
            if (rc != V3DBA_OK)
            {
               std::fprintf(stderr, "v3dba_minimize failed: %s\n", v3dba_error_string(rc));
               return;
            }
            unpack(Kb, R, T, D);
            status = r.status;
            currentIteration = r.iterations;
            lambda = r.lambda;
            lastResult = r;
         }

         int precision;          //!< V3DBA_PRECISION_MIXED (default) or V3DBA_PRECISION_FP64
         int lastError;          //!< V3DBA_OK or the error code of the last C-ABI call
         v3dba_result lastResult;

      protected:
         // The points are read and written in place: a vector<Vector3d> is 3 doubles per element.
         double* points() { return _Xs.empty() ? 0 : _Xs[0].begin(); }

         void pack(std::vector<double>& Kb, std::vector<double>& R, std::vector<double>& T,
                   std::vector<double>& D) const
         {
            int const N = _cams.size();
            R.resize(9 * (size_t)N); T.resize(3 * (size_t)N);
            Kb.resize(_model == V3DBA_MODEL_COMMON ? 9 : 9 * (size_t)N);
            for (int i = 0; i < N; ++i)
            {
               Matrix3x3d const& Ri = _cams[i].getRotation();
               Vector3d const& Ti = _cams[i].getTranslation();
               Matrix3x3d const& Ki = _cams[i].getIntrinsic();
               for (int r = 0; r < 3; ++r)
               {
                  T[3 * i + r] = Ti[r];
                  for (int c = 0; c < 3; ++c)
                  {
                     R[9 * i + 3 * r + c] = Ri[r][c];
                     if (_model != V3DBA_MODEL_COMMON) Kb[9 * i + 3 * r + c] = Ki[r][c];
                  }
               }
            }
            if (_model == V3DBA_MODEL_COMMON)
               for (int r = 0; r < 3; ++r)
                  for (int c = 0; c < 3; ++c) Kb[3 * r + c] = (*_K)[r][c];
            D.clear();
            if (_model == V3DBA_MODEL_COMMON)
            {
               D.push_back(_distortion->k1); D.push_back(_distortion->k2);
               D.push_back(_distortion->p1); D.push_back(_distortion->p2);
            }
            else if (_model == V3DBA_MODEL_VARYING)
               for (int i = 0; i < N; ++i)
               {
                  StdDistortionFunction const& d = (*_distortions)[i];
                  D.push_back(d.k1); D.push_back(d.k2); D.push_back(d.p1); D.push_back(d.p2);
               }
         }

         void unpack(std::vector<double> const& Kb, std::vector<double> const& R, std::vector<double> const& T,
                     std::vector<double> const& D)
         {
            int const N = _cams.size();
            for (int i = 0; i < N; ++i)
            {
               Matrix3x3d Ri;
               Vector3d Ti;
               for (int r = 0; r < 3; ++r)
               {
                  Ti[r] = T[3 * i + r];
                  for (int c = 0; c < 3; ++c) Ri[r][c] = R[9 * i + 3 * r + c];
               }
               _cams[i].setRotation(Ri);
               _cams[i].setTranslation(Ti);
               if (_model == V3DBA_MODEL_VARYING)
               {
                  Matrix3x3d Ki;
                  for (int r = 0; r < 3; ++r)
                     for (int c = 0; c < 3; ++c) Ki[r][c] = Kb[9 * i + 3 * r + c];
                  _cams[i].setIntrinsic(Ki);
                  StdDistortionFunction& d = (*_distortions)[i];
                  d.k1 = D[4 * i]; d.k2 = D[4 * i + 1]; d.p1 = D[4 * i + 2]; d.p2 = D[4 * i + 3];
               }
            }
            if (_model == V3DBA_MODEL_COMMON)
            {
               for (int r = 0; r < 3; ++r)
                  for (int c = 0; c < 3; ++c) (*_K)[r][c] = Kb[3 * r + c];
               _distortion->k1 = D[0]; _distortion->k2 = D[1]; _distortion->p1 = D[2]; _distortion->p2 = D[3];
            }
         }

         int const _model, _mode;
         vector<CameraMatrix>& _cams;
         vector<Vector3d>& _Xs;
         Matrix3x3d* _K;
         StdDistortionFunction* _distortion;
         vector<StdDistortionFunction>* _distortions;
         v3dba_handle _handle;
         int _nnA, _nnB, _nnC;
   }; // end struct MetricBundleOptimizerBase

   struct StdMetricBundleOptimizer : public MetricBundleOptimizerBase
   {
         StdMetricBundleOptimizer(double inlierThreshold,
                                  vector<CameraMatrix>& cams,
                                  vector<Vector3d>& Xs,
                                  vector<Vector2d> const& measurements,
                                  vector<int> const& corrspondingView,
                                  vector<int> const& corrspondingPoint)
            : MetricBundleOptimizerBase(V3DBA_MODEL_STD, 0, inlierThreshold, cams, Xs, measurements,
                                        corrspondingView, corrspondingPoint, 0, 0, 0)
         { }
   };

   struct CommonInternalsMetricBundleOptimizer : public MetricBundleOptimizerBase
   {
         static int globalParamDimensionFromMode(int mode)
         {
            int dA = 6, dC = 0;
            v3dba_dims(V3DBA_MODEL_COMMON, mode, &dA, &dC);
            return dC;
         }

         CommonInternalsMetricBundleOptimizer(int mode,
                                              double inlierThreshold,
                                              Matrix3x3d& K,
                                              StdDistortionFunction& distortion,
                                              vector<CameraMatrix>& cams,
                                              vector<Vector3d>& Xs,
                                              vector<Vector2d> const& measurements,
                                              vector<int> const& corrspondingView,
                                              vector<int> const& corrspondingPoint)
            : MetricBundleOptimizerBase(V3DBA_MODEL_COMMON, mode, inlierThreshold, cams, Xs, measurements,
                                        corrspondingView, corrspondingPoint, &K, &distortion, 0)
         { }
   };

   //! The name the B200 design uses for the shared-intrinsics distortion adjuster.
   typedef CommonInternalsMetricBundleOptimizer StdDistortionMetricBundleOptimizer;

   struct VaryingInternalsMetricBundleOptimizer : public MetricBundleOptimizerBase
   {
         static int extParamDimensionFromMode(int mode)
         {
            int dA = 6, dC = 0;
            v3dba_dims(V3DBA_MODEL_VARYING, mode, &dA, &dC);
            return dA - 6;
         }

         VaryingInternalsMetricBundleOptimizer(int mode,
                                               double inlierThreshold,
                                               std::vector<StdDistortionFunction>& distortions,
                                               vector<CameraMatrix>& cams,
                                               vector<Vector3d>& Xs,
                                               vector<Vector2d> const& measurements,
                                               vector<int> const& corrspondingView,
                                               vector<int> const& corrspondingPoint)
            : MetricBundleOptimizerBase(V3DBA_MODEL_VARYING, mode, inlierThreshold, cams, Xs, measurements,
                                        corrspondingView, corrspondingPoint, 0, 0, &distortions)
         { }
   };

   //! Normalizes the 3D points and camera centers to zero mean and unit overall norm for the
   //! duration of a scope (ScopedBundleExtrinsicNormalizer, v3d_metricbundle.h:325-383).
   struct ScopedBundleExtrinsicNormalizer
   {
         ScopedBundleExtrinsicNormalizer(vector<CameraMatrix>& cameras, vector<Vector3d>& Xs)
            : _cameras(cameras), _Xs(Xs)
         {
            int const N = cameras.size(), M = Xs.size();
            vector<Vector3d> centers(N);
            for (int i = 0; i < N; ++i) centers[i] = cameras[i].cameraCenter();
            for (int r = 0; r < 3; ++r) _mean[r] = 0.0;
            for (int i = 0; i < N; ++i) for (int r = 0; r < 3; ++r) _mean[r] += centers[i][r];
            for (int j = 0; j < M; ++j) for (int r = 0; r < 3; ++r) _mean[r] += Xs[j][r];
            for (int r = 0; r < 3; ++r) _mean[r] /= double(N + M);
            double sq = 0.0;
            for (int i = 0; i < N; ++i) for (int r = 0; r < 3; ++r) { centers[i][r] -= _mean[r]; sq += centers[i][r] * centers[i][r]; }
            for (int j = 0; j < M; ++j) for (int r = 0; r < 3; ++r) { Xs[j][r] -= _mean[r]; sq += Xs[j][r] * Xs[j][r]; }
            _scale = std::sqrt(sq);
            double const inv = 1.0 / _scale;
            for (int i = 0; i < N; ++i) { for (int r = 0; r < 3; ++r) centers[i][r] *= inv; cameras[i].setCameraCenter(centers[i]); }
            for (int j = 0; j < M; ++j) for (int r = 0; r < 3; ++r) Xs[j][r] *= inv;
         }

         ~ScopedBundleExtrinsicNormalizer()
         {
            int const N = _cameras.size(), M = _Xs.size();
            for (int i = 0; i < N; ++i)
            {
               Vector3d c = _cameras[i].cameraCenter();
               for (int r = 0; r < 3; ++r) c[r] = c[r] * _scale + _mean[r];
               _cameras[i].setCameraCenter(c);
            }
            for (int j = 0; j < M; ++j) for (int r = 0; r < 3; ++r) _Xs[j][r] = _Xs[j][r] * _scale + _mean[r];
         }

      protected:
         vector<CameraMatrix>& _cameras;
         vector<Vector3d>& _Xs;
         Vector3d _mean;
         double _scale;
   };

   //! Scales every camera's K and its measurements to unit focal length for the duration of a
   //! scope (ScopedBundleIntrinsicNormalizer, v3d_metricbundle.h:386-443).
   struct ScopedBundleIntrinsicNormalizer
   {
         ScopedBundleIntrinsicNormalizer(vector<CameraMatrix>& cameras, vector<Vector2d>& measurements,
                                         vector<int> const& correspondingView)
            : _cameras(cameras), _measurements(measurements), _correspondingView(correspondingView),
              _savedFs(cameras.size())
         {
            for (size_t i = 0; i < cameras.size(); ++i)
            {
               Matrix3x3d KK = cameras[i].getIntrinsic();
               double const f = KK[0][0];
               _savedFs[i] = f;
               for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) KK[r][c] /= f;
               KK[2][2] = 1.0;
               cameras[i].setIntrinsic(KK);
            }
            for (size_t k = 0; k < measurements.size(); ++k)
            {
               double const f = _savedFs[correspondingView[k]];
               measurements[k][0] /= f; measurements[k][1] /= f;
            }
         }

         ~ScopedBundleIntrinsicNormalizer()
         {
            for (size_t i = 0; i < _cameras.size(); ++i)
            {
               Matrix3x3d KK = _cameras[i].getIntrinsic();
               for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) KK[r][c] *= _savedFs[i];
               KK[2][2] = 1.0;
               _cameras[i].setIntrinsic(KK);
            }
            for (size_t k = 0; k < _measurements.size(); ++k)
            {
               double const f = _savedFs[_correspondingView[k]];
               _measurements[k][0] *= f; _measurements[k][1] *= f;
            }
         }

      protected:
         vector<CameraMatrix>& _cameras;
         vector<Vector2d>& _measurements;
         vector<int> const& _correspondingView;
         vector<double> _savedFs;
   };

} // end namespace V3D

#endif
