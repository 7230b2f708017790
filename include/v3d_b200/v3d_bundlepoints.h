// -*- C++ -*-
// B200 BundlePointStructure with the members, constructor and createPointStructure of the
// reference's struct (Geometry/v3d_mviewutilities.h:132-205), built on the GPU through
// v3dba_bundle_point_structure / v3dba_create_point_structure (v3dba.h).
//
// The reference defines its struct inline in v3d_mviewutilities.h, next to TriangulatedPoint and
// PointMeasurement, which a caller keeps using; this header declares the same struct in
// V3D::B200.  A caller switches with
//     #include "v3d_b200/v3d_bundlepoints.h"
//     using V3D::B200::BundlePointStructure;
// and links libv3dba.so.  The members and their contents are the reference's, bit for bit.  The
// reference has no error path; here a GPU-side error leaves the members empty (or the
// reconstruction unchanged), is reported on stderr and kept in `lastError` (V3DBA_OK == 0).
#ifndef V3D_B200_BUNDLEPOINTS_H
#define V3D_B200_BUNDLEPOINTS_H

#include <cstdio>
#include <vector>

#include "Geometry/v3d_mviewutilities.h"

#include "v3dba.h"

namespace V3D
{
   namespace B200
   {
      struct BundlePointStructure
      {
            BundlePointStructure() : lastError(V3DBA_OK) { }

            BundlePointStructure(std::vector<TriangulatedPoint> const& reconstruction,
                                 int nRequiredMeasurements = 2)
               : lastError(V3DBA_OK)
            {
               std::vector<int> ptr, view, id;
               std::vector<double> pos;
               std::vector<float> mpos;
               flatten(reconstruction, ptr, pos, view, id, mpos);
               int const n = (int)reconstruction.size(), K = ptr.back();
               std::vector<double> pts(3 * (size_t)n), meas(2 * (size_t)K);
               std::vector<int> ids(K), cv(K), cp(K), xs(n);
               int np = 0, nm = 0;
               lastError = v3dba_bundle_point_structure(n, ptr.data(), pos.data(), view.data(), id.data(), mpos.data(),
                                                        nRequiredMeasurements, &np, &nm, pts.data(), meas.data(),
                                                        ids.data(), cv.data(), cp.data(), xs.data());
               if (lastError != V3DBA_OK)
               {
                  std::fprintf(stderr, "v3dba_bundle_point_structure failed: %s\n", v3dba_error_string(lastError));
                  return;
               }
               points3d.resize(np);
               xsIndices.assign(xs.begin(), xs.begin() + np);
               for (int i = 0; i < np; ++i) points3d[i] = makeVector3(pts[3*i], pts[3*i+1], pts[3*i+2]);
               measurements.resize(nm);
               for (int k = 0; k < nm; ++k) measurements[k] = makeVector2(meas[2*k], meas[2*k+1]);
               measurementIds.assign(ids.begin(), ids.begin() + nm);
               correspondingView.assign(cv.begin(), cv.begin() + nm);
               correspondingPoint.assign(cp.begin(), cp.begin() + nm);
            }

            void createPointStructure(std::vector<TriangulatedPoint>& reconstruction, bool createFromScratch = true)
            {
               int const M = (int)points3d.size(), K = (int)measurements.size();
               std::vector<double> pts(3 * (size_t)M), meas(2 * (size_t)K);
               for (int i = 0; i < M; ++i)
                  for (int c = 0; c < 3; ++c) pts[3*i+c] = points3d[i][c];
               for (int k = 0; k < K; ++k)
               {
                  meas[2*k] = measurements[k][0];
                  meas[2*k+1] = measurements[k][1];
               }
               std::vector<int> ptr, view, id;
               std::vector<double> pos;
               std::vector<float> mpos;
               if (createFromScratch)
               {
                  ptr.assign(M + 1, 0);
                  pos.assign(3 * (size_t)M, 0.0);
                  view.assign(K, 0);
                  id.assign(K, 0);
                  mpos.assign(2 * (size_t)K, 0.0f);
               }
               else
               {
                  flatten(reconstruction, ptr, pos, view, id, mpos);
               }
               int const n = createFromScratch ? M : (int)reconstruction.size();
               lastError = v3dba_create_point_structure(createFromScratch ? 1 : 0, M, K, pts.data(), meas.data(),
                                                        measurementIds.data(), correspondingView.data(),
                                                        correspondingPoint.data(), xsIndices.data(), n, ptr.data(),
                                                        pos.data(), view.data(), id.data(), mpos.data());
               if (lastError != V3DBA_OK)
               {
                  std::fprintf(stderr, "v3dba_create_point_structure failed: %s\n", v3dba_error_string(lastError));
                  return;
               }
               reconstruction.resize(n);
               for (int j = 0; j < n; ++j)
               {
                  TriangulatedPoint& X = reconstruction[j];
                  X.pos = makeVector3(pos[3*j], pos[3*j+1], pos[3*j+2]);
                  X.measurements.resize(ptr[j+1] - ptr[j]);
                  for (int m = ptr[j]; m < ptr[j+1]; ++m)
                  {
                     PointMeasurement& pm = X.measurements[m - ptr[j]];
                     pm.view = view[m];
                     pm.id = id[m];
                     pm.pos[0] = mpos[2*m];
                     pm.pos[1] = mpos[2*m+1];
                  }
               }
            }

            std::vector<Vector3d> points3d;
            std::vector<Vector2d> measurements;
            std::vector<int>      measurementIds;
            std::vector<int>      correspondingView;
            std::vector<int>      correspondingPoint;
            std::vector<int>      xsIndices;
            int                   lastError;

         private:
            static void flatten(std::vector<TriangulatedPoint> const& rec, std::vector<int>& ptr, std::vector<double>& pos,
                                std::vector<int>& view, std::vector<int>& id, std::vector<float>& mpos)
            {
               ptr.assign(1, 0);
               pos.clear();
               view.clear();
               id.clear();
               mpos.clear();
               for (size_t j = 0; j < rec.size(); ++j)
               {
                  for (int c = 0; c < 3; ++c) pos.push_back(rec[j].pos[c]);
                  for (size_t k = 0; k < rec[j].measurements.size(); ++k)
                  {
                     PointMeasurement const& pm = rec[j].measurements[k];
                     view.push_back(pm.view);
                     id.push_back(pm.id);
                     mpos.push_back(pm.pos[0]);
                     mpos.push_back(pm.pos[1]);
                  }
                  ptr.push_back((int)view.size());
               }
               if (pos.empty()) pos.push_back(0.0);   // data() of an empty vector may be NULL
               if (view.empty()) { view.push_back(0); id.push_back(0); mpos.push_back(0.0f); mpos.push_back(0.0f); }
            }
      }; // end struct BundlePointStructure
   } // end namespace B200
} // end namespace V3D

#endif
