// A reference-style caller of V3D::B200::BundlePointStructure (include/v3d_b200/v3d_bundlepoints.h)
// checked against the reference's own inline struct (V3D/include/Geometry/v3d_mviewutilities.h:
// 132-205) on seeded random reconstructions: every member after the constructor, and the
// reconstruction after createPointStructure in both branches, must be identical.
//
//   points_demo [seed]      exit code 0 when every comparison holds
#include "v3d_b200/v3d_bundlepoints.h"

#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace V3D;

static unsigned long long g_state = 1;
static unsigned next_u32() {
   g_state = g_state * 6364136223846793005ull + 1442695040888963407ull;
   return (unsigned)(g_state >> 33);
}
static double uniform(double a, double b) { return a + (b - a) * (next_u32() / 4294967296.0); }

static std::vector<TriangulatedPoint> random_reconstruction(int n, int max_len) {
   std::vector<TriangulatedPoint> rec(n);
   for (int j = 0; j < n; ++j) {
      rec[j].pos = makeVector3(uniform(-10, 10), uniform(-10, 10), uniform(5, 50));
      int const len = (int)(next_u32() % (unsigned)(max_len + 1));
      for (int k = 0; k < len; ++k) {
         PointMeasurement m;
         m.view = (int)(next_u32() % 40u);
         m.id = (int)(next_u32() % 100000u) - 1;
         m.pos[0] = (float)uniform(0, 640);
         m.pos[1] = (float)uniform(0, 480);
         rec[j].measurements.push_back(m);
      }
   }
   return rec;
}

template <typename A, typename B>
static bool same_members(A const& a, B const& b) {
   if (a.points3d.size() != b.points3d.size() || a.measurements.size() != b.measurements.size()) return false;
   for (size_t i = 0; i < a.points3d.size(); ++i)
      for (int c = 0; c < 3; ++c)
         if (a.points3d[i][c] != b.points3d[i][c]) return false;
   for (size_t k = 0; k < a.measurements.size(); ++k)
      for (int c = 0; c < 2; ++c)
         if (a.measurements[k][c] != b.measurements[k][c]) return false;
   return a.measurementIds == b.measurementIds && a.correspondingView == b.correspondingView &&
          a.correspondingPoint == b.correspondingPoint && a.xsIndices == b.xsIndices;
}

static bool same_reconstruction(std::vector<TriangulatedPoint> const& a, std::vector<TriangulatedPoint> const& b) {
   if (a.size() != b.size()) return false;
   for (size_t j = 0; j < a.size(); ++j) {
      for (int c = 0; c < 3; ++c)
         if (a[j].pos[c] != b[j].pos[c]) return false;
      if (a[j].measurements.size() != b[j].measurements.size()) return false;
      for (size_t k = 0; k < a[j].measurements.size(); ++k) {
         PointMeasurement const &p = a[j].measurements[k], &q = b[j].measurements[k];
         if (p.view != q.view || p.id != q.id || p.pos[0] != q.pos[0] || p.pos[1] != q.pos[1]) return false;
      }
   }
   return true;
}

int main(int argc, char** argv) {
   g_state = argc > 1 ? std::strtoull(argv[1], 0, 10) : 1;
   int failures = 0, cases = 0;
   int const sizes[][2] = {{0, 0}, {7, 0}, {500, 1}, {2000, 8}, {100, 200}};
   int const thresholds[] = {-1, 0, 1, 2, 5};
   for (auto const& sz : sizes) {
      std::vector<TriangulatedPoint> const rec = random_reconstruction(sz[0], sz[1]);
      for (int nreq : thresholds) {
         ++cases;
         V3D::BundlePointStructure ref(rec, nreq);
         V3D::B200::BundlePointStructure gpu(rec, nreq);
         if (gpu.lastError != V3DBA_OK || !same_members(ref, gpu)) {
            std::printf("constructor differs: n=%d len<=%d nRequired=%d\n", sz[0], sz[1], nreq);
            ++failures;
            continue;
         }
         // the adjusted values an optimizer would write
         for (size_t i = 0; i < ref.points3d.size(); ++i) {
            ref.points3d[i][0] += 0.25;
            gpu.points3d[i][0] += 0.25;
         }
         for (size_t k = 0; k < ref.measurements.size(); ++k) {
            ref.measurements[k][1] = ref.measurements[k][1] / 3.0;
            gpu.measurements[k][1] = gpu.measurements[k][1] / 3.0;
         }
         for (int scratch = 0; scratch < 2; ++scratch) {
            std::vector<TriangulatedPoint> a = rec, b = rec;
            ref.createPointStructure(a, scratch != 0);
            gpu.createPointStructure(b, scratch != 0);
            if (gpu.lastError != V3DBA_OK || !same_reconstruction(a, b)) {
               std::printf("createPointStructure(%s) differs: n=%d len<=%d nRequired=%d\n",
                           scratch ? "true" : "false", sz[0], sz[1], nreq);
               ++failures;
            }
         }
      }
   }
   std::printf("%d cases, %d failures\n", cases, failures);
   return failures ? 1 : 0;
}
