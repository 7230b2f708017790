// -*- C++ -*-
// B200 rotation averaging with the signature of the reference's V3D::refineConsistentRotations
// (Geometry/v3d_mviewutilities.h:359-362; implementation V3D/src/Geometry/v3d_mviewutilities.cpp:
// 470-611, the SparseRotationOptimizer LM with maxIterations = 200), running on the GPU through
// v3dba_refine_consistent_rotations (v3dba.h).
//
// The reference defines the function in v3d_mviewutilities.cpp next to many other multi-view
// utilities a caller keeps using, so this header does not redefine V3D::refineConsistentRotations
// (two definitions would clash at link time).  It declares the same function in V3D::B200; a
// caller switches with
//     #include "v3d_b200/v3d_mviewutilities.h"
//     using V3D::B200::refineConsistentRotations;   // or call V3D::B200::refineConsistentRotations
// and links libv3dba.so.  Arguments, their meaning and the in-place update of `rotations` are
// the reference's.  The reference has no error path; on a GPU-side error (CUDA failure, a view
// index out of range, a non-finite input) this version leaves `rotations` unchanged, reports the
// error on stderr and returns the v3dba error code (V3DBA_OK == 0) instead of void.
#ifndef V3D_B200_MVIEWUTILITIES_H
#define V3D_B200_MVIEWUTILITIES_H

#include <cstdio>
#include <utility>
#include <vector>

#include "Math/v3d_linear.h"

#include "v3dba.h"

namespace V3D
{
   namespace B200
   {
      static_assert(sizeof(Matrix3x3d) == 9 * sizeof(double), "Matrix3x3d must be 9 packed doubles");
      static_assert(sizeof(std::pair<int, int>) == 2 * sizeof(int), "pair<int, int> must be two packed ints");

      inline int
      refineConsistentRotations(int const nViews,
                                std::vector<Matrix3x3d> const& relativeRotations,
                                std::vector<std::pair<int, int> > const& viewPairs,
                                std::vector<Matrix3x3d>& rotations)
      {
         if ((int)rotations.size() < nViews || relativeRotations.size() < viewPairs.size())
         {
            std::fprintf(stderr, "refineConsistentRotations: fewer rotations than views or pairs\n");
            return V3DBA_ERR_INVALID_ARGUMENT;
         }
         v3dba_options opts;
         v3dba_default_options(&opts);
         opts.max_iterations = 200;   // SparseRotationOptimizer's constructor
         std::vector<double> R(9 * (size_t)nViews);
         for (int i = 0; i < nViews; ++i)
            for (int r = 0; r < 3; ++r)
               for (int c = 0; c < 3; ++c) R[9 * i + 3 * r + c] = rotations[i][r][c];
         int const nPairs = (int)viewPairs.size();
         int const rc = v3dba_refine_consistent_rotations(
            nViews, nPairs, nPairs ? relativeRotations[0][0] : 0,
            nPairs ? reinterpret_cast<int32_t const*>(&viewPairs[0]) : 0, R.data(), &opts, 0);
         if (rc != V3DBA_OK)
         {
            std::fprintf(stderr, "v3dba_refine_consistent_rotations failed: %s\n", v3dba_error_string(rc));
            return rc;
         }
         for (int i = 0; i < nViews; ++i)
            for (int r = 0; r < 3; ++r)
               for (int c = 0; c < 3; ++c) rotations[i][r][c] = R[9 * i + 3 * r + c];
         return V3DBA_OK;
      }
   } // end namespace B200
} // end namespace V3D

#endif
