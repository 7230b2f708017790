// A reference-style caller of V3D::B200::refineConsistentRotations: builds the reference's
// Matrix3x3d / pair<int, int> containers and calls the function as the reference's own entry
// point is called (V3D/include/Geometry/v3d_mviewutilities.h:359-362).
//
//   rotations_demo <graph.bin> <out.bin>
//
// graph.bin (little-endian): int32 nViews, nPairs; float64 rel[9 nPairs]; int32 pairs[2 nPairs];
// float64 R[9 nViews].  out.bin: int32 rc; float64 R[9 nViews].
#include "v3d_b200/v3d_mviewutilities.h"

#include <cstdio>
#include <vector>

using namespace V3D;

template <typename T>
static bool rd(FILE* f, T* p, size_t n) { return fread(p, sizeof(T), n, f) == n; }

int main(int argc, char** argv)
{
   if (argc < 3) { fprintf(stderr, "usage: rotations_demo graph.bin out.bin\n"); return 2; }
   FILE* f = fopen(argv[1], "rb");
   if (!f) return 2;
   int n[2];
   if (!rd(f, n, 2)) return 2;
   int const N = n[0], P = n[1];
   std::vector<double> rel(9 * (size_t)P), R(9 * (size_t)N);
   std::vector<int> pr(2 * (size_t)P);
   if (!rd(f, rel.data(), rel.size()) || !rd(f, pr.data(), pr.size()) || !rd(f, R.data(), R.size())) return 2;
   fclose(f);

   std::vector<Matrix3x3d> relativeRotations(P), rotations(N);
   std::vector<std::pair<int, int> > viewPairs(P);
   for (int k = 0; k < P; ++k)
   {
      for (int r = 0; r < 3; ++r)
         for (int c = 0; c < 3; ++c) relativeRotations[k][r][c] = rel[9 * k + 3 * r + c];
      viewPairs[k] = std::make_pair(pr[2 * k], pr[2 * k + 1]);
   }
   for (int i = 0; i < N; ++i)
      for (int r = 0; r < 3; ++r)
         for (int c = 0; c < 3; ++c) rotations[i][r][c] = R[9 * i + 3 * r + c];

   int const rc = B200::refineConsistentRotations(N, relativeRotations, viewPairs, rotations);

   FILE* o = fopen(argv[2], "wb");
   if (!o) return 2;
   fwrite(&rc, sizeof(int), 1, o);
   for (int i = 0; i < N; ++i)
      for (int r = 0; r < 3; ++r) fwrite(rotations[i][r], sizeof(double), 3, o);
   fclose(o);
   return rc == V3DBA_OK ? 0 : 1;
}
