// A reference-style caller of the rig bundle adjuster: builds the reference's containers
// (Matrix3x3d rig rotations, Vector3d translations and points, CameraMatrix rig cameras) and
// calls StereoMetricBundleOptimizer as the reference declares it
// (V3D/include/Geometry/v3d_stereobundle.h:26-56), with only the include swapped.
//
//   stereo_demo <scene.bin> <out.bin>
//
// scene.bin (little-endian): int32 N, M, K, L, maxIterations, precision, nnA, nnB;
// float64 inlierThreshold; float64 R[9N], T[3N], X[3M], meas[2K], rigK[9L], rigR[9L], rigT[3L];
// int32 view[K], point[K], sub[K].  out.bin: int32 status, iterations; float64 R, T, X.
#include "v3d_b200/v3d_stereobundle.h"

#include <cstdio>
#include <vector>

using namespace V3D;

template <typename T>
static bool rd(FILE* f, T* p, size_t n) { return fread(p, sizeof(T), n, f) == n; }

int main(int argc, char** argv)
{
   if (argc < 3) { fprintf(stderr, "usage: stereo_demo scene.bin out.bin\n"); return 2; }
   FILE* f = fopen(argv[1], "rb");
   if (!f) return 2;
   int hdr[8];
   double thr;
   if (!rd(f, hdr, 8) || !rd(f, &thr, 1)) return 2;
   int const N = hdr[0], M = hdr[1], K = hdr[2], L = hdr[3];
   std::vector<double> R(9 * N), T(3 * N), X(3 * M), meas(2 * K), rK(9 * L), rR(9 * L), rT(3 * L);
   std::vector<int> view(K), point(K), sub(K);
   if (!rd(f, R.data(), R.size()) || !rd(f, T.data(), T.size()) || !rd(f, X.data(), X.size()) ||
       !rd(f, meas.data(), meas.size()) || !rd(f, rK.data(), rK.size()) || !rd(f, rR.data(), rR.size()) ||
       !rd(f, rT.data(), rT.size()) || !rd(f, view.data(), K) || !rd(f, point.data(), K) || !rd(f, sub.data(), K))
      return 2;
   fclose(f);

   std::vector<Matrix3x3d> rotations(N);
   std::vector<Vector3d> translations(N), Xs(M);
   std::vector<CameraMatrix> rig(L);
   std::vector<Vector2d> measurements(K);
   for (int i = 0; i < N; ++i)
   {
      for (int r = 0; r < 3; ++r)
      {
         translations[i][r] = T[3 * i + r];
         for (int c = 0; c < 3; ++c) rotations[i][r][c] = R[9 * i + 3 * r + c];
      }
   }
   for (int j = 0; j < M; ++j) Xs[j] = Vector3d(X[3 * j], X[3 * j + 1], X[3 * j + 2]);
   for (int l = 0; l < L; ++l)
   {
      Matrix3x3d Kl, Rl;
      for (int r = 0; r < 3; ++r)
         for (int c = 0; c < 3; ++c) { Kl[r][c] = rK[9 * l + 3 * r + c]; Rl[r][c] = rR[9 * l + 3 * r + c]; }
      rig[l] = CameraMatrix(Kl, Rl, Vector3d(rT[3 * l], rT[3 * l + 1], rT[3 * l + 2]));
   }
   for (int k = 0; k < K; ++k) { measurements[k][0] = meas[2 * k]; measurements[k][1] = meas[2 * k + 1]; }

   StereoMetricBundleOptimizer opt(thr, rotations, translations, rig, Xs, measurements, view, point, sub);
   opt.setNonvaryingCounts(hdr[6], hdr[7], 0);
   opt.maxIterations = hdr[4];
   opt.precision = hdr[5];
   opt.minimize();
   if (opt.lastError != V3DBA_OK) return 1;

   FILE* o = fopen(argv[2], "wb");
   if (!o) return 2;
   int const st[2] = { opt.status, opt.currentIteration };
   fwrite(st, sizeof(int), 2, o);
   for (int i = 0; i < N; ++i)
      for (int r = 0; r < 3; ++r) fwrite(rotations[i][r], sizeof(double), 3, o);
   for (int i = 0; i < N; ++i) fwrite(translations[i].begin(), sizeof(double), 3, o);
   for (int j = 0; j < M; ++j) fwrite(Xs[j].begin(), sizeof(double), 3, o);
   fclose(o);
   return 0;
}
