// -*- C++ -*-
// Drop-in replacement of the reference header Geometry/v3d_stereobundle.h: the rig bundle
// adjuster StereoMetricBundleOptimizer, running on the B200 through the C-ABI of v3dba.h
// (V3DBA_MODEL_STEREO).
//
// A caller keeps its code and swaps
//     #include "Geometry/v3d_stereobundle.h"
// for
//     #include "v3d_b200/v3d_stereobundle.h"
// and links libv3dba.so instead of compiling v3d_stereobundle.cpp.  The class keeps the
// reference's name, constructor signature (V3D/include/Geometry/v3d_stereobundle.h:26-56),
// public LevenbergOptimizerCommon fields and minimize(); it holds references to the caller's rig
// rotations, translations and points and updates them in place.  The rig cameras stay fixed.
//
// Differences, all deliberate:
//   * maxIterations defaults to 50 (LevenbergOptimizerCommon's value); the reference leaves the
//     SparseLevenbergOptimizer field uninitialised (v3d_optimization.h:382).
//   * Fixed poses / points (setNonvaryingCounts) are handled exactly (see v3d_metricbundle.h).
//   * GPU-side errors are reported on stderr and in lastError, with status
//     LEVENBERG_OPTIMIZER_TIMEOUT and the parameters untouched.
#ifndef V3D_B200_STEREOBUNDLE_H
#define V3D_B200_STEREOBUNDLE_H

#include <cstdio>
#include <vector>

#include "Geometry/v3d_cameramatrix.h"
#include "Math/v3d_linear.h"
#include "Math/v3d_optimization.h"

#include "v3dba.h"

namespace V3D
{
   using std::vector;

   struct StereoMetricBundleOptimizer : public LevenbergOptimizerCommon
   {
         StereoMetricBundleOptimizer(double inlierThreshold,
                                     vector<Matrix3x3d>& rotations,
                                     vector<Vector3d>& translations,
                                     vector<CameraMatrix> const& rigCameras,
                                     vector<Vector3d>& Xs,
                                     vector<Vector2d> const& measurements,
                                     vector<int> const& corrspondingView,
                                     vector<int> const& corrspondingPoint,
                                     vector<int> const& correspondingSubCamera)
            : LevenbergOptimizerCommon(), precision(V3DBA_PRECISION_MIXED), lastError(V3DBA_OK),
              _rotations(rotations), _translations(translations), _Xs(Xs), _handle(0), _nnA(0), _nnB(0)
         {
            static_assert(sizeof(Vector2d) == 2 * sizeof(double), "Vector2d must be two packed doubles");
            static_assert(sizeof(Vector3d) == 3 * sizeof(double), "Vector3d must be three packed doubles");
            static_assert(sizeof(Matrix3x3d) == 9 * sizeof(double), "Matrix3x3d must be 9 packed doubles");
            int const N = rotations.size(), L = rigCameras.size(), Kn = measurements.size();
            std::vector<double> rigK(9 * (size_t)L), rigR(9 * (size_t)L), rigT(3 * (size_t)L);
            for (int l = 0; l < L; ++l)
               for (int r = 0; r < 3; ++r)
               {
                  rigT[3 * l + r] = rigCameras[l].getTranslation()[r];
                  for (int c = 0; c < 3; ++c)
                  {
                     rigK[9 * l + 3 * r + c] = rigCameras[l].getIntrinsic()[r][c];
                     rigR[9 * l + 3 * r + c] = rigCameras[l].getRotation()[r][c];
                  }
               }
            v3dba_problem p = v3dba_problem();
            p.model = V3DBA_MODEL_STEREO; p.mode = 0;
            p.n_cameras = N; p.n_points = Xs.size(); p.n_measurements = Kn;
            p.inlier_threshold = inlierThreshold;
            p.R = N ? rotations[0][0] : 0;
            p.T = N ? translations[0].begin() : 0;
            p.X = points();
            p.measurements = Kn ? measurements[0].begin() : 0;
            p.view = corrspondingView.data(); p.point = corrspondingPoint.data();
            p.n_rig_cameras = L;
            p.rig_K = rigK.data(); p.rig_R = rigR.data(); p.rig_T = rigT.data();
            p.subcamera = correspondingSubCamera.data();
            lastError = v3dba_create(&p, &_handle);
            if (lastError != V3DBA_OK)
            {
               std::fprintf(stderr, "v3dba_create failed: %s\n", v3dba_error_string(lastError));
               _handle = 0;
            }
         }

         virtual ~StereoMetricBundleOptimizer() { if (_handle) v3dba_destroy(_handle); }

         void setNonvaryingCounts(int nNonvaryingA, int nNonvaryingB, int nNonvaryingC)
         {
            _nnA = nNonvaryingA; _nnB = nNonvaryingB; (void)nNonvaryingC;
         }

         void getNonvaryingCounts(int& nNonvaryingA, int& nNonvaryingB, int& nNonvaryingC) const
         {
            nNonvaryingA = _nnA; nNonvaryingB = _nnB; nNonvaryingC = 0;
         }

         void minimize()
         {
            status = LEVENBERG_OPTIMIZER_TIMEOUT;
            if (!_handle) return;
            // rotations, translations and points are passed and returned in place
            double* R = _rotations.empty() ? 0 : _rotations[0][0];
            double* T = _translations.empty() ? 0 : _translations[0].begin();
            int rc = v3dba_set_params(_handle, 0, R, T, 0, points());
            if (rc == V3DBA_OK) rc = v3dba_set_nonvarying(_handle, _nnA, _nnB, 0);
            if (rc == V3DBA_OK) rc = v3dba_set_lambda(_handle, lambda);
            v3dba_options o;
            v3dba_default_options(&o);
            o.tau = tau; o.max_iterations = maxIterations;
            o.gradient_threshold = gradientThreshold; o.update_threshold = updateThreshold;
            o.verbosity = optimizerVerbosenessLevel;
            o.precision = precision;
            v3dba_result r;
            if (rc == V3DBA_OK) rc = v3dba_minimize(_handle, &o, &r);
            if (rc == V3DBA_OK) rc = v3dba_get_params(_handle, 0, R, T, 0, points());
            lastError = rc;
            if (rc != V3DBA_OK)
            {
               std::fprintf(stderr, "v3dba_minimize failed: %s\n", v3dba_error_string(rc));
               return;
            }
            status = r.status;
            currentIteration = r.iterations;
            lambda = r.lambda;
            lastResult = r;
         }

         int precision;          //!< V3DBA_PRECISION_MIXED (default) or V3DBA_PRECISION_FP64
         int lastError;          //!< V3DBA_OK or the error code of the last C-ABI call
         v3dba_result lastResult;

      protected:
         double* points() { return _Xs.empty() ? 0 : _Xs[0].begin(); }

         vector<Matrix3x3d>& _rotations;
         vector<Vector3d>& _translations;
         vector<Vector3d>& _Xs;
         v3dba_handle _handle;
         int _nnA, _nnB;
   }; // end struct StereoMetricBundleOptimizer

} // end namespace V3D

#endif
