// A reference-style caller of the drop-in header: it builds V3D::CameraMatrix / Vector3d inputs
// and calls the optimizer exactly as the reference's pipeline stages do
// (SfM/generate_triples/src/generate_triples.cpp:404-412), with only the include swapped.
//
//   shim_demo <scene.bin> <out.bin>
//
// scene.bin (little-endian): int32 model, mode, N, M, K, maxIterations, precision, nnA, nnB, nnC;
// float64 inlierThreshold; float64 K[9 or 9N]; R[9N]; T[3N]; dist[4 or 4N or 0]; X[3M];
// meas[2K]; int32 view[K], point[K].
// out.bin: int32 status, iterations; float64 K, R, T, dist, X in the same layout.
#include "v3d_b200/v3d_metricbundle.h"

#include <cstdio>
#include <vector>

using namespace V3D;

template <typename T>
static bool rd(FILE* f, T* p, size_t n) { return fread(p, sizeof(T), n, f) == n; }

int main(int argc, char** argv)
{
   if (argc < 3) { fprintf(stderr, "usage: shim_demo scene.bin out.bin\n"); return 2; }
   FILE* f = fopen(argv[1], "rb");
   if (!f) return 2;
   int hdr[10];
   double thr;
   if (!rd(f, hdr, 10) || !rd(f, &thr, 1)) return 2;
   int const model = hdr[0], mode = hdr[1], N = hdr[2], M = hdr[3], K = hdr[4];
   int const nK = model == V3DBA_MODEL_COMMON ? 9 : 9 * N;
   int const nD = model == V3DBA_MODEL_COMMON ? 4 : (model == V3DBA_MODEL_VARYING ? 4 * N : 0);
   std::vector<double> Kb(nK), R(9 * N), T(3 * N), D(nD), X(3 * M), meas(2 * K);
   std::vector<int> view(K), point(K);
   if (!rd(f, Kb.data(), nK) || !rd(f, R.data(), 9 * N) || !rd(f, T.data(), 3 * N) ||
       (nD && !rd(f, D.data(), nD)) || !rd(f, X.data(), 3 * M) || !rd(f, meas.data(), 2 * K) ||
       !rd(f, view.data(), K) || !rd(f, point.data(), K))
      return 2;
   fclose(f);

   std::vector<CameraMatrix> cams(N);
   Matrix3x3d Kshared;
   for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) Kshared[r][c] = Kb[3 * r + c];
   for (int i = 0; i < N; ++i)
   {
      Matrix3x3d Ki, Ri;
      Vector3d Ti;
      for (int r = 0; r < 3; ++r)
      {
         Ti[r] = T[3 * i + r];
         for (int c = 0; c < 3; ++c)
         {
            Ri[r][c] = R[9 * i + 3 * r + c];
            Ki[r][c] = model == V3DBA_MODEL_COMMON ? Kshared[r][c] : Kb[9 * i + 3 * r + c];
         }
      }
      cams[i] = CameraMatrix(Ki, Ri, Ti);
   }
   std::vector<Vector3d> Xs(M);
   for (int j = 0; j < M; ++j) Xs[j] = Vector3d(X[3 * j], X[3 * j + 1], X[3 * j + 2]);
   std::vector<Vector2d> ms(K);
   for (int k = 0; k < K; ++k) { ms[k][0] = meas[2 * k]; ms[k][1] = meas[2 * k + 1]; }
   StdDistortionFunction dist;
   std::vector<StdDistortionFunction> dists(model == V3DBA_MODEL_VARYING ? N : 0);
   if (model == V3DBA_MODEL_COMMON) { dist.k1 = D[0]; dist.k2 = D[1]; dist.p1 = D[2]; dist.p2 = D[3]; }
   for (int i = 0; i < (int)dists.size(); ++i)
   { dists[i].k1 = D[4 * i]; dists[i].k2 = D[4 * i + 1]; dists[i].p1 = D[4 * i + 2]; dists[i].p2 = D[4 * i + 3]; }

   int status = -1, iters = -1;
   {
      MetricBundleOptimizerBase* opt = 0;
      if (model == V3DBA_MODEL_STD)
         opt = new StdMetricBundleOptimizer(thr, cams, Xs, ms, view, point);
      else if (model == V3DBA_MODEL_COMMON)
         opt = new CommonInternalsMetricBundleOptimizer(mode, thr, Kshared, dist, cams, Xs, ms, view, point);
      else
         opt = new VaryingInternalsMetricBundleOptimizer(mode, thr, dists, cams, Xs, ms, view, point);
      opt->setNonvaryingCounts(hdr[7], hdr[8], hdr[9]);
      V3D::optimizerVerbosenessLevel = 0;
      opt->tau = 1e-3;
      opt->maxIterations = hdr[5];
      opt->precision = hdr[6];
      opt->minimize();
      status = opt->status;
      iters = opt->currentIteration;
      if (opt->lastError != V3DBA_OK) { fprintf(stderr, "error %d\n", opt->lastError); return 1; }
      delete opt;
   }

   FILE* o = fopen(argv[2], "wb");
   if (!o) return 2;
   int st[2] = {status, iters};
   fwrite(st, sizeof(int), 2, o);
   for (int i = 0; i < N; ++i)
      for (int r = 0; r < 3; ++r)
         for (int c = 0; c < 3; ++c)
            Kb[(model == V3DBA_MODEL_COMMON ? 0 : 9 * i) + 3 * r + c] =
               model == V3DBA_MODEL_COMMON ? Kshared[r][c] : cams[i].getIntrinsic()[r][c];
   for (int i = 0; i < N; ++i)
      for (int r = 0; r < 3; ++r)
      {
         T[3 * i + r] = cams[i].getTranslation()[r];
         for (int c = 0; c < 3; ++c) R[9 * i + 3 * r + c] = cams[i].getRotation()[r][c];
      }
   if (model == V3DBA_MODEL_COMMON) { D[0] = dist.k1; D[1] = dist.k2; D[2] = dist.p1; D[3] = dist.p2; }
   for (int i = 0; i < (int)dists.size(); ++i)
   { D[4 * i] = dists[i].k1; D[4 * i + 1] = dists[i].k2; D[4 * i + 2] = dists[i].p1; D[4 * i + 3] = dists[i].p2; }
   for (int j = 0; j < M; ++j) for (int r = 0; r < 3; ++r) X[3 * j + r] = Xs[j][r];
   fwrite(Kb.data(), sizeof(double), nK, o);
   fwrite(R.data(), sizeof(double), 9 * N, o);
   fwrite(T.data(), sizeof(double), 3 * N, o);
   if (nD) fwrite(D.data(), sizeof(double), nD, o);
   fwrite(X.data(), sizeof(double), 3 * M, o);
   fclose(o);
   return 0;
}
