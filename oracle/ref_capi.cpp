// TEST INFRASTRUCTURE ONLY -- never linked into, or called by, the product library.
//
// A C-ABI around the reference's own sparse LM bundle adjuster, compiled from the
// untouched reference sources (see oracle/Makefile).  It lets tests and the bench's
// CPU baseline drive the reference optimizer classes on flat structure-of-arrays
// inputs:
//   * V3D::StdMetricBundleOptimizer             (V3D/include/Geometry/v3d_metricbundle.h:107-136)
//   * V3D::CommonInternalsMetricBundleOptimizer (V3D/include/Geometry/v3d_metricbundle.h:150-238)
//   * V3D::VaryingInternalsMetricBundleOptimizer(V3D/include/Geometry/v3d_metricbundle.h:242-320)
// all running V3D::SparseLevenbergOptimizer::minimize (V3D/src/Math/v3d_optimization.cpp:719-1250),
// and the rotation averaging V3D::refineConsistentRotations (V3D/src/Geometry/
// v3d_mviewutilities.cpp:470-613), which runs the same minimize() on SparseRotationOptimizer,
// and V3D::StereoMetricBundleOptimizer (V3D/include/Geometry/v3d_stereobundle.h:22-163),
// and the triplet stage around the triplet adjustment (SfM/generate_triples/src/
// generate_triples.cpp:380-415).
//
// Parameter layout (row-major, doubles), shared with the product C-ABI:
//   K    : model 0/2 -> nCams*9 per-camera intrinsics; model 1 -> 9 (the shared K)
//   R    : nCams*9,  T : nCams*3,  X : nPoints*3
//   dist : model 1 -> 4 {k1,k2,p1,p2}; model 2 -> nCams*4; model 0 -> unused
//   meas : nObs*2,  view/point : nObs (0-based)

#include "Geometry/v3d_metricbundle.h"
#include "Geometry/v3d_mviewutilities.h"
#include "Geometry/v3d_stereobundle.h"

#include <cmath>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

using namespace V3D;

namespace
{
   enum { MODEL_STD = 0, MODEL_COMMON = 1, MODEL_VARYING = 2 };

   struct Trace
   {
      double* cost; double* lambda; int* iter; int cap; int len;
      int nRejected;
   };

   // Records the weighted cost each time the optimizer relinearizes: fillWeights is
   // called once per relinearization (v3d_optimization.cpp:785), before the lambda
   // for that iteration is initialised.
   template <typename Opt>
   struct Traced : public Opt
   {
      template <typename... Args>
      Traced(Trace* tr, Args&&... args) : Opt(std::forward<Args>(args)...), _tr(tr) { }

      virtual void fillWeights(VectorArray<double> const& residual, Vector<double>& w)
      {
         Opt::fillWeights(residual, w);
         if (_tr && _tr->len < _tr->cap)
         {
            double err = 0.0;
            for (unsigned k = 0; k < w.size(); ++k)
               err += w[k] * w[k] * (residual[k][0] * residual[k][0] + residual[k][1] * residual[k][1]);
            _tr->cost[_tr->len] = err;
            _tr->lambda[_tr->len] = this->lambda;
            _tr->iter[_tr->len] = this->currentIteration;
         }
         if (_tr) ++_tr->len;
      }

      virtual void restoreAllParameters()
      {
         Opt::restoreAllParameters();
         if (_tr) ++_tr->nRejected;
      }

      Trace* _tr;
   };

   struct Scene
   {
      std::vector<CameraMatrix> cams;
      std::vector<Vector3d> Xs;
      std::vector<Vector2d> meas;
      std::vector<int> view, point;
      Matrix3x3d Kshared;
      StdDistortionFunction dist;
      std::vector<StdDistortionFunction> dists;
   };

   void loadMat3(double const* p, Matrix3x3d& M)
   {
      for (int r = 0; r < 3; ++r)
         for (int c = 0; c < 3; ++c) M[r][c] = p[3 * r + c];
   }

   void storeMat3(Matrix3x3d const& M, double* p)
   {
      for (int r = 0; r < 3; ++r)
         for (int c = 0; c < 3; ++c) p[3 * r + c] = M[r][c];
   }

   void loadDist(double const* p, StdDistortionFunction& d)
   {
      d.k1 = p[0]; d.k2 = p[1]; d.p1 = p[2]; d.p2 = p[3];
   }

   void storeDist(StdDistortionFunction const& d, double* p)
   {
      p[0] = d.k1; p[1] = d.k2; p[2] = d.p1; p[3] = d.p2;
   }

   void buildScene(Scene& s, int model, int nCams, int nPoints, int nObs,
                   double const* K, double const* R, double const* T, double const* dist,
                   double const* X, double const* meas, int const* view, int const* point)
   {
      s.cams.resize(nCams);
      if (model == MODEL_COMMON) loadMat3(K, s.Kshared);
      for (int i = 0; i < nCams; ++i)
      {
         Matrix3x3d Ki, Ri;
         Vector3d Ti;
         if (model == MODEL_COMMON) Ki = s.Kshared; else loadMat3(K + 9 * i, Ki);
         loadMat3(R + 9 * i, Ri);
         Ti[0] = T[3 * i]; Ti[1] = T[3 * i + 1]; Ti[2] = T[3 * i + 2];
         s.cams[i] = CameraMatrix(Ki, Ri, Ti);
      }
      s.Xs.resize(nPoints);
      for (int j = 0; j < nPoints; ++j)
         s.Xs[j] = Vector3d(X[3 * j], X[3 * j + 1], X[3 * j + 2]);
      s.meas.resize(nObs);
      for (int k = 0; k < nObs; ++k)
      {
         s.meas[k][0] = meas[2 * k];
         s.meas[k][1] = meas[2 * k + 1];
      }
      s.view.assign(view, view + nObs);
      s.point.assign(point, point + nObs);
      if (model == MODEL_COMMON) loadDist(dist, s.dist);
      if (model == MODEL_VARYING)
      {
         s.dists.resize(nCams);
         for (int i = 0; i < nCams; ++i) loadDist(dist + 4 * i, s.dists[i]);
      }
   }

   void exportScene(Scene const& s, int model, double* K, double* R, double* T, double* dist, double* X)
   {
      int const nCams = s.cams.size();
      for (int i = 0; i < nCams; ++i)
      {
         if (model != MODEL_COMMON) storeMat3(s.cams[i].getIntrinsic(), K + 9 * i);
         storeMat3(s.cams[i].getRotation(), R + 9 * i);
         Vector3d const& Ti = s.cams[i].getTranslation();
         T[3 * i] = Ti[0]; T[3 * i + 1] = Ti[1]; T[3 * i + 2] = Ti[2];
      }
      if (model == MODEL_COMMON) { storeMat3(s.Kshared, K); storeDist(s.dist, dist); }
      if (model == MODEL_VARYING)
         for (int i = 0; i < nCams; ++i) storeDist(s.dists[i], dist + 4 * i);
      for (size_t j = 0; j < s.Xs.size(); ++j)
      {
         X[3 * j] = s.Xs[j][0]; X[3 * j + 1] = s.Xs[j][1]; X[3 * j + 2] = s.Xs[j][2];
      }
   }

   bool validModel(int model, int mode)
   {
      if (model < MODEL_STD || model > MODEL_VARYING) return false;
      if (model != MODEL_STD && (mode < FULL_BUNDLE_NO_ROTATIONS || mode > FULL_BUNDLE_RADIAL_TANGENTIAL))
         return false;
      return true;
   }

   template <typename Opt>
   void runMinimize(Opt& opt, int nnA, int nnB, int nnC, double tau, int maxIterations,
                    int* status, int* iterations, double* lambda)
   {
      opt.setNonvaryingCounts(nnA, nnB, nnC);
      opt.tau = tau;
      opt.maxIterations = maxIterations;
      opt.minimize();
      *status = opt.status;
      *iterations = opt.currentIteration;
      *lambda = opt.lambda;
   }
} // end namespace <>

extern "C"
{

int v3dref_param_dims(int model, int mode, int* dA, int* dC)
{
   if (!validModel(model, mode)) return -1;
   *dA = 6; *dC = 0;
   if (model == MODEL_COMMON) *dC = CommonInternalsMetricBundleOptimizer::globalParamDimensionFromMode(mode);
   if (model == MODEL_VARYING) *dA = 6 + VaryingInternalsMetricBundleOptimizer::extParamDimensionFromMode(mode);
   return 0;
}

// Runs the reference minimize(). Parameters are updated in place.  The optional trace
// (any pointer may be NULL when traceCap == 0) receives one (iteration, lambda, cost)
// entry per relinearization.
int v3dref_minimize(int model, int mode, int nCams, int nPoints, int nObs, double inlierThreshold,
                    double* K, double* R, double* T, double* dist, double* X,
                    double const* meas, int const* view, int const* point,
                    int nnA, int nnB, int nnC, double tau, int maxIterations, int verbosity,
                    int* status, int* iterations, double* lambda,
                    double* traceCost, double* traceLambda, int* traceIter, int traceCap,
                    int* traceLen, int* nRejected)
{
   if (!validModel(model, mode)) return -1;
   Scene s;
   buildScene(s, model, nCams, nPoints, nObs, K, R, T, dist, X, meas, view, point);
   Trace tr = { traceCost, traceLambda, traceIter, traceCap, 0, 0 };
   V3D::optimizerVerbosenessLevel = verbosity;

   if (model == MODEL_STD)
   {
      Traced<StdMetricBundleOptimizer> opt(&tr, inlierThreshold, s.cams, s.Xs, s.meas, s.view, s.point);
      runMinimize(opt, nnA, nnB, nnC, tau, maxIterations, status, iterations, lambda);
   }
   else if (model == MODEL_COMMON)
   {
      Traced<CommonInternalsMetricBundleOptimizer> opt(&tr, mode, inlierThreshold, s.Kshared, s.dist,
                                                       s.cams, s.Xs, s.meas, s.view, s.point);
      runMinimize(opt, nnA, nnB, nnC, tau, maxIterations, status, iterations, lambda);
   }
   else
   {
      Traced<VaryingInternalsMetricBundleOptimizer> opt(&tr, mode, inlierThreshold, s.dists,
                                                        s.cams, s.Xs, s.meas, s.view, s.point);
      runMinimize(opt, nnA, nnB, nnC, tau, maxIterations, status, iterations, lambda);
   }
   V3D::optimizerVerbosenessLevel = 0;
   exportScene(s, model, K, R, T, dist, X);
   if (traceLen) *traceLen = tr.len;
   if (nRejected) *nRejected = tr.nRejected;
   return 0;
}

// Per-observation residual e_k = proj - m_k, Huber weight w_k and the raw (unweighted)
// Jacobian blocks A_k (2 x dA), B_k (2 x 3), C_k (2 x dC), all row-major, evaluated by the
// reference's own evalResidual / fillWeights / fillJacobians.  Any output may be NULL.
int v3dref_linearize(int model, int mode, int nCams, int nPoints, int nObs, double inlierThreshold,
                     double const* K, double const* R, double const* T, double const* dist,
                     double const* X, double const* meas, int const* view, int const* point,
                     double* e, double* w, double* A, double* B, double* C)
{
   int dA, dC;
   if (v3dref_param_dims(model, mode, &dA, &dC) != 0) return -1;
   Scene s;
   buildScene(s, model, nCams, nPoints, nObs, K, R, T, dist, X, meas, view, point);

   SparseLevenbergOptimizer* opt = 0;
   if (model == MODEL_STD)
      opt = new StdMetricBundleOptimizer(inlierThreshold, s.cams, s.Xs, s.meas, s.view, s.point);
   else if (model == MODEL_COMMON)
      opt = new CommonInternalsMetricBundleOptimizer(mode, inlierThreshold, s.Kshared, s.dist,
                                                     s.cams, s.Xs, s.meas, s.view, s.point);
   else
      opt = new VaryingInternalsMetricBundleOptimizer(mode, inlierThreshold, s.dists,
                                                      s.cams, s.Xs, s.meas, s.view, s.point);

   VectorArray<double> res(nObs, 2);
   Vector<double> weights(nObs);
   opt->evalResidual(res);
   opt->fillWeights(res, weights);

   Matrix<double> Ak(2, dA), Bk(2, 3), Ck(2, dC > 0 ? dC : 1);
   for (int k = 0; k < nObs; ++k)
   {
      if (e) { e[2 * k] = res[k][0]; e[2 * k + 1] = res[k][1]; }
      if (w) w[k] = weights[k];
      if (A || B || C)
      {
         makeZeroMatrix(Ak); makeZeroMatrix(Bk); makeZeroMatrix(Ck);
         opt->fillJacobians(Ak, Bk, Ck, view[k], point[k], k);
         for (int r = 0; r < 2; ++r)
         {
            if (A) for (int c = 0; c < dA; ++c) A[(2 * k + r) * dA + c] = Ak[r][c];
            if (B) for (int c = 0; c < 3; ++c) B[(2 * k + r) * 3 + c] = Bk[r][c];
            if (C) for (int c = 0; c < dC; ++c) C[(2 * k + r) * dC + c] = Ck[r][c];
         }
      }
   }
   delete opt;
   return 0;
}

// Final cost as the harness defines it: sum_k |w_k e_k|^2 with the Huber weights
// recomputed at the given parameters (v3d_metricbundle.h:49-57, v3d_optimization.cpp:784-789).
double v3dref_cost(int model, int mode, int nCams, int nPoints, int nObs, double inlierThreshold,
                   double const* K, double const* R, double const* T, double const* dist,
                   double const* X, double const* meas, int const* view, int const* point)
{
   std::vector<double> e(2 * (size_t)nObs), w(nObs);
   if (v3dref_linearize(model, mode, nCams, nPoints, nObs, inlierThreshold, K, R, T, dist, X,
                        meas, view, point, e.data(), w.data(), 0, 0, 0) != 0)
      return -1.0;
   double err = 0.0;
   for (int k = 0; k < nObs; ++k)
      err += w[k] * w[k] * (e[2 * k] * e[2 * k] + e[2 * k + 1] * e[2 * k + 1]);
   return err;
}

// V3D::refineConsistentRotations on nViews row-major 3x3 rotations (updated in place), nPairs
// relative rotations and view pairs (2 ints each).  The function sets optimizerVerbosenessLevel
// to 1, so minimize() prints "|residual|^2 = <err>" once per relinearization
// (v3d_optimization.cpp:791); std::cout is redirected to a buffer at full precision for the
// call and those values are returned as the cost trace (traceErr[0..*traceLen), up to traceCap).
int v3dref_refine_rotations(int nViews, int nPairs, double const* relR, int const* pairs, double* R,
                            double* traceErr, int traceCap, int* traceLen)
{
   std::vector<Matrix3x3d> rel(nPairs), rots(nViews);
   std::vector<std::pair<int, int> > vp(nPairs);
   for (int k = 0; k < nPairs; ++k)
   {
      for (int r = 0; r < 3; ++r)
         for (int c = 0; c < 3; ++c) rel[k][r][c] = relR[9 * k + 3 * r + c];
      vp[k] = std::make_pair(pairs[2 * k], pairs[2 * k + 1]);
   }
   for (int i = 0; i < nViews; ++i)
      for (int r = 0; r < 3; ++r)
         for (int c = 0; c < 3; ++c) rots[i][r][c] = R[9 * i + 3 * r + c];

   std::ostringstream captured;
   captured.precision(17);
   std::streambuf* saved = std::cout.rdbuf(captured.rdbuf());
   std::streamsize savedPrec = std::cout.precision(17);
   refineConsistentRotations(nViews, rel, vp, rots);
   std::cout.precision(savedPrec);
   std::cout.rdbuf(saved);
   V3D::optimizerVerbosenessLevel = 0;

   for (int i = 0; i < nViews; ++i)
      for (int r = 0; r < 3; ++r)
         for (int c = 0; c < 3; ++c) R[9 * i + 3 * r + c] = rots[i][r][c];

   int len = 0;
   std::istringstream lines(captured.str());
   std::string line;
   std::string const tag = "|residual|^2 = ";
   while (std::getline(lines, line))
   {
      size_t const at = line.find(tag);
      if (at == std::string::npos) continue;
      if (len < traceCap && traceErr) traceErr[len] = std::strtod(line.c_str() + at + tag.size(), 0);
      ++len;
   }
   if (traceLen) *traceLen = len;
   return 0;
}

// StereoMetricBundleOptimizer: nPoses rig poses (R 9, T 3 each; updated in place), nPoints
// points (updated in place), nRig fixed rig cameras (K 9, R 9, T 3), measurements with view,
// point and rig camera indices.  Same outputs as v3dref_minimize.
int v3dref_minimize_stereo(int nPoses, int nPoints, int nObs, int nRig, double inlierThreshold,
                           double* R, double* T, double* X, double const* meas, int const* view,
                           int const* point, int const* sub, double const* rigK, double const* rigR,
                           double const* rigT, int nnA, int nnB, double tau, int maxIterations,
                           int* status, int* iterations, double* lambda,
                           double* traceCost, double* traceLambda, int* traceIter, int traceCap,
                           int* traceLen, int* nRejected)
{
   std::vector<Matrix3x3d> rotations(nPoses);
   std::vector<Vector3d> translations(nPoses), Xs(nPoints);
   std::vector<CameraMatrix> rig(nRig);
   std::vector<Vector2d> ms(nObs);
   for (int i = 0; i < nPoses; ++i)
   {
      loadMat3(R + 9 * i, rotations[i]);
      translations[i] = Vector3d(T[3 * i], T[3 * i + 1], T[3 * i + 2]);
   }
   for (int j = 0; j < nPoints; ++j) Xs[j] = Vector3d(X[3 * j], X[3 * j + 1], X[3 * j + 2]);
   for (int l = 0; l < nRig; ++l)
   {
      Matrix3x3d Kl, Rl;
      loadMat3(rigK + 9 * l, Kl);
      loadMat3(rigR + 9 * l, Rl);
      rig[l] = CameraMatrix(Kl, Rl, Vector3d(rigT[3 * l], rigT[3 * l + 1], rigT[3 * l + 2]));
   }
   for (int k = 0; k < nObs; ++k) { ms[k][0] = meas[2 * k]; ms[k][1] = meas[2 * k + 1]; }
   std::vector<int> vv(view, view + nObs), pp(point, point + nObs), ss(sub, sub + nObs);

   Trace tr = { traceCost, traceLambda, traceIter, traceCap, 0, 0 };
   V3D::optimizerVerbosenessLevel = 0;
   Traced<StereoMetricBundleOptimizer> opt(&tr, inlierThreshold, rotations, translations, rig, Xs, ms, vv, pp, ss);
   runMinimize(opt, nnA, nnB, 0, tau, maxIterations, status, iterations, lambda);

   for (int i = 0; i < nPoses; ++i)
   {
      storeMat3(rotations[i], R + 9 * i);
      T[3 * i] = translations[i][0]; T[3 * i + 1] = translations[i][1]; T[3 * i + 2] = translations[i][2];
   }
   for (int j = 0; j < nPoints; ++j) { X[3 * j] = Xs[j][0]; X[3 * j + 1] = Xs[j][1]; X[3 * j + 2] = Xs[j][2]; }
   if (traceLen) *traceLen = tr.len;
   if (nRejected) *nRejected = tr.nRejected;
   return 0;
}

// Residuals, Huber weights and raw Jacobians (A 2x6, B 2x3 per observation) of the stereo model
// from the reference's evalResidual / fillWeights / fillJacobians.  Any output may be NULL.
int v3dref_linearize_stereo(int nPoses, int nPoints, int nObs, int nRig, double inlierThreshold,
                            double const* R, double const* T, double const* X, double const* meas,
                            int const* view, int const* point, int const* sub, double const* rigK,
                            double const* rigR, double const* rigT, double* e, double* w, double* A, double* B)
{
   std::vector<Matrix3x3d> rotations(nPoses);
   std::vector<Vector3d> translations(nPoses), Xs(nPoints);
   std::vector<CameraMatrix> rig(nRig);
   std::vector<Vector2d> ms(nObs);
   for (int i = 0; i < nPoses; ++i)
   {
      loadMat3(R + 9 * i, rotations[i]);
      translations[i] = Vector3d(T[3 * i], T[3 * i + 1], T[3 * i + 2]);
   }
   for (int j = 0; j < nPoints; ++j) Xs[j] = Vector3d(X[3 * j], X[3 * j + 1], X[3 * j + 2]);
   for (int l = 0; l < nRig; ++l)
   {
      Matrix3x3d Kl, Rl;
      loadMat3(rigK + 9 * l, Kl);
      loadMat3(rigR + 9 * l, Rl);
      rig[l] = CameraMatrix(Kl, Rl, Vector3d(rigT[3 * l], rigT[3 * l + 1], rigT[3 * l + 2]));
   }
   for (int k = 0; k < nObs; ++k) { ms[k][0] = meas[2 * k]; ms[k][1] = meas[2 * k + 1]; }
   std::vector<int> vv(view, view + nObs), pp(point, point + nObs), ss(sub, sub + nObs);
   StereoMetricBundleOptimizer opt(inlierThreshold, rotations, translations, rig, Xs, ms, vv, pp, ss);

   VectorArray<double> res(nObs, 2);
   Vector<double> weights(nObs);
   opt.evalResidual(res);
   opt.fillWeights(res, weights);
   Matrix<double> Ak(2, 6), Bk(2, 3), Ck(2, 1);
   for (int k = 0; k < nObs; ++k)
   {
      if (e) { e[2 * k] = res[k][0]; e[2 * k + 1] = res[k][1]; }
      if (w) w[k] = weights[k];
      if (A || B)
      {
         makeZeroMatrix(Ak); makeZeroMatrix(Bk);
         opt.fillJacobians(Ak, Bk, Ck, view[k], point[k], k);
         for (int r = 0; r < 2; ++r)
         {
            if (A) for (int c = 0; c < 6; ++c) A[(2 * k + r) * 6 + c] = Ak[r][c];
            if (B) for (int c = 0; c < 3; ++c) B[(2 * k + r) * 3 + c] = Bk[r][c];
         }
      }
   }
   return 0;
}

// The triplet stage of SfM/generate_triples/src/generate_triples.cpp:380-415 for one triplet,
// with the reference's own triangulateLinear (V3D/include/Geometry/v3d_mviewutilities.h:296-303),
// BundlePointStructure (:132-205) and StdMetricBundleOptimizer.  filterTripleModel
// (generate_triples.cpp:44-81) lives in the application file, which needs the reference's
// database layer to compile; it is restated here on the reference's own types (Vector2f,
// norm_L2, CameraMatrix::projectPoint), so its float arithmetic is the reference's.
// Outputs: verdict (0 accepted, 1 too few points, 2 too many dropped), surviving track count,
// the adjustment's status / iterations / last relinearisation cost, cameras after it, every
// track's point (refined for surviving tracks of accepted triplets, else the triangulation) and
// the filter's decision per measurement.
int v3dref_triplet_stage(double const* R, double const* T, double const* focal, int nTracks,
                         int const* trackPtr, int const* view, float const* pos, double maxError,
                         int minPoints, double minRatio, double inlierThreshold, double tau, int maxIterations,
                         int* verdict, int* nSurvived, int* status, int* iterations, double* cost,
                         double* Rout, double* Tout, double* Xout, unsigned char* keptOut)
{
   std::vector<CameraMatrix> tripleCams(3);
   Matrix3x3d I;
   makeIdentityMatrix(I);
   for (int i = 0; i < 3; ++i)
   {
      Matrix3x3d Ri;
      loadMat3(R + 9 * i, Ri);
      tripleCams[i].setIntrinsic(I);
      tripleCams[i].setRotation(Ri);
      tripleCams[i].setTranslation(Vector3d(T[3 * i], T[3 * i + 1], T[3 * i + 2]));
   }
   std::vector<TriangulatedPoint> tripleModel(nTracks);
   for (int j = 0; j < nTracks; ++j)
      for (int m = trackPtr[j]; m < trackPtr[j + 1]; ++m)
         tripleModel[j].measurements.push_back(
            PointMeasurement(makeVector2<float>(pos[2 * m], pos[2 * m + 1]), view[m], m));

   int const nPointsBefore = tripleModel.size();
   for (int j = 0; j < nPointsBefore; ++j)
      tripleModel[j].pos = triangulateLinear(tripleCams, tripleModel[j].measurements);

   // filterTripleModel, generate_triples.cpp:44-81 (restated; see above)
   std::vector<int> survivors;
   for (int j = 0; j < nPointsBefore; ++j)
   {
      TriangulatedPoint& X = tripleModel[j];
      std::vector<PointMeasurement> ms;
      for (size_t k = 0; k < X.measurements.size(); ++k)
      {
         PointMeasurement const& m = X.measurements[k];
         Vector2d p = tripleCams[m.view].projectPoint(X.pos);
         Vector2f pp = makeVector2<float>(p[0], p[1]);
         double const err = focal[m.view] * norm_L2(pp - m.pos);
         bool const keep = err < maxError;
         keptOut[m.id] = keep ? 1 : 0;
         if (keep) ms.push_back(m);
      }
      X.measurements = ms;
      if (X.measurements.size() >= 3) survivors.push_back(j);
   }
   for (int j = 0; j < nPointsBefore; ++j)
      for (int r = 0; r < 3; ++r) Xout[3 * j + r] = tripleModel[j].pos[r];
   std::vector<TriangulatedPoint> model;
   for (size_t q = 0; q < survivors.size(); ++q) model.push_back(tripleModel[survivors[q]]);

   *nSurvived = model.size();
   *verdict = 0;
   if ((int)model.size() < minPoints) *verdict = 1;
   else if (double(model.size()) < minRatio * nPointsBefore) *verdict = 2;
   *status = 0; *iterations = 0; *cost = 0.0;
   if (*verdict == 0)
   {
      BundlePointStructure bundleStruct(model);
      double tc[1024], tl[1024];
      int ti[1024];
      Trace tr = { tc, tl, ti, 1024, 0, 0 };
      Traced<StdMetricBundleOptimizer> opt(&tr, inlierThreshold, tripleCams, bundleStruct.points3d,
                                           bundleStruct.measurements, bundleStruct.correspondingView,
                                           bundleStruct.correspondingPoint);
      V3D::optimizerVerbosenessLevel = 0;
      opt.tau = tau;
      opt.maxIterations = maxIterations;
      opt.minimize();
      *status = opt.status;
      *iterations = opt.currentIteration;
      *cost = tr.len > 0 ? tc[std::min(tr.len, 1024) - 1] : 0.0;
      bundleStruct.createPointStructure(model);
      for (size_t q = 0; q < survivors.size(); ++q)
         for (int r = 0; r < 3; ++r) Xout[3 * survivors[q] + r] = model[q].pos[r];
   }
   for (int i = 0; i < 3; ++i)
   {
      storeMat3(tripleCams[i].getRotation(), Rout + 9 * i);
      Vector3d const& Ti = tripleCams[i].getTranslation();
      Tout[3 * i] = Ti[0]; Tout[3 * i + 1] = Ti[1]; Tout[3 * i + 2] = Ti[2];
   }
   return 0;
}

// ---- BundlePointStructure (V3D/include/Geometry/v3d_mviewutilities.h:132-205) ----------------
// Tracks in the flat form of v3dba.h: track j = TriangulatedPoint j with pos trackPos[3j..] and
// measurements trackPtr[j] .. trackPtr[j + 1] - 1 (view, id, float position).

static std::vector<TriangulatedPoint>
tracksToReconstruction(int nTracks, int const* trackPtr, double const* trackPos, int const* view, int const* id,
                       float const* pos)
{
   std::vector<TriangulatedPoint> rec(nTracks);
   for (int j = 0; j < nTracks; ++j)
   {
      rec[j].pos = makeVector3(trackPos[3*j], trackPos[3*j+1], trackPos[3*j+2]);
      for (int m = trackPtr[j]; m < trackPtr[j+1]; ++m)
      {
         PointMeasurement pm;
         pm.view = view ? view[m] : 0;
         pm.id = id ? id[m] : -1;
         pm.pos[0] = pos[2*m];
         pm.pos[1] = pos[2*m+1];
         rec[j].measurements.push_back(pm);
      }
   }
   return rec;
}

static void
reconstructionToTracks(std::vector<TriangulatedPoint> const& rec, int* trackPtr, double* trackPos, int* view, int* id,
                       float* pos)
{
   int m = 0;
   trackPtr[0] = 0;
   for (size_t j = 0; j < rec.size(); ++j)
   {
      for (int c = 0; c < 3; ++c) trackPos[3*j+c] = rec[j].pos[c];
      for (size_t k = 0; k < rec[j].measurements.size(); ++k, ++m)
      {
         if (view) view[m] = rec[j].measurements[k].view;
         if (id) id[m] = rec[j].measurements[k].id;
         pos[2*m] = rec[j].measurements[k].pos[0];
         pos[2*m+1] = rec[j].measurements[k].pos[1];
      }
      trackPtr[j+1] = m;
   }
}

int v3dref_bundle_point_structure(int nTracks, int const* trackPtr, double const* trackPos, int const* view,
                                  int const* id, float const* pos, int nRequired, int* nPoints, int* nMeasurements,
                                  double* points3d, double* measurements, int* measurementIds, int* correspondingView,
                                  int* correspondingPoint, int* xsIndices)
{
   std::vector<TriangulatedPoint> const rec = tracksToReconstruction(nTracks, trackPtr, trackPos, view, id, pos);
   BundlePointStructure bps(rec, nRequired);
   *nPoints = (int)bps.points3d.size();
   *nMeasurements = (int)bps.measurements.size();
   for (size_t i = 0; i < bps.points3d.size(); ++i)
   {
      for (int c = 0; c < 3; ++c) points3d[3*i+c] = bps.points3d[i][c];
      xsIndices[i] = bps.xsIndices[i];
   }
   for (size_t k = 0; k < bps.measurements.size(); ++k)
   {
      measurements[2*k] = bps.measurements[k][0];
      measurements[2*k+1] = bps.measurements[k][1];
      measurementIds[k] = bps.measurementIds[k];
      correspondingView[k] = bps.correspondingView[k];
      correspondingPoint[k] = bps.correspondingPoint[k];
   }
   return 0;
}

int v3dref_create_point_structure(int fromScratch, int nPoints, int nMeasurements, double const* points3d,
                                  double const* measurements, int const* measurementIds, int const* correspondingView,
                                  int const* correspondingPoint, int const* xsIndices, int nTracks, int* trackPtr,
                                  double* trackPos, int* view, int* id, float* pos)
{
   BundlePointStructure bps;
   for (int i = 0; i < nPoints; ++i)
   {
      bps.points3d.push_back(makeVector3(points3d[3*i], points3d[3*i+1], points3d[3*i+2]));
      if (xsIndices) bps.xsIndices.push_back(xsIndices[i]);
   }
   for (int k = 0; k < nMeasurements; ++k)
   {
      bps.measurements.push_back(makeVector2(measurements[2*k], measurements[2*k+1]));
      bps.measurementIds.push_back(measurementIds ? measurementIds[k] : -1);
      bps.correspondingView.push_back(correspondingView ? correspondingView[k] : 0);
      bps.correspondingPoint.push_back(correspondingPoint ? correspondingPoint[k] : 0);
   }
   std::vector<TriangulatedPoint> rec;
   if (!fromScratch) rec = tracksToReconstruction(nTracks, trackPtr, trackPos, view, id, pos);
   bps.createPointStructure(rec, fromScratch != 0);
   reconstructionToTracks(rec, trackPtr, trackPos, view, id, pos);
   return 0;
}

} // extern "C"

