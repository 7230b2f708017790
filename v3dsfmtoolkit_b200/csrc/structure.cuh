// Device construction of a problem's structure (structure.cu).
#pragma once

#include <cstdint>
#include <functional>
#include <vector>

#include "common.cuh"

namespace v3dba {

// Allocates `bytes` of device memory that the caller owns (the handle's buffers).
using DevAlloc = std::function<int(void**, size_t)>;

struct DeviceStructure {
  // device, allocated through the DevAlloc
  int* o_orig = nullptr;   // [K] caller's index of each point-major observation
  int* o_pt = nullptr;     // [K] point of each observation
  int* o_cam = nullptr;    // [K] camera of each observation
  double* o_meas = nullptr;   // [2K]
  int* p_ptr = nullptr;    // [M+1] observations of each point
  int* c_ptr = nullptr;    // [N+1] observations of each camera ...
  int* c_obs = nullptr;    // [K]   ... in point-major order
  int* b_i = nullptr;      // [nb] camera-pair blocks (i <= l), (i, l) order
  int* b_l = nullptr;
  int* b_ptr = nullptr;    // [nb+1] pairs of each block
  int* pr_k = nullptr;     // [P] observation of camera i in each pair
  int* pr_m = nullptr;     // [P] observation of camera l
  int64_t P = 0;
  // host copies of the small arrays
  std::vector<int> h_c_ptr, h_b_i, h_b_l, h_b_ptr;
};

// Builds the structure of `p` (validated indices) on the device, on stream `st`.
int build_structure_device(const v3dba_problem* p, const DevAlloc& alloc, cudaStream_t st, DeviceStructure& S);

// Stable grouping of n items by device int keys in [0, nv): perm[t] is the t-th item in key
// order (input order among equal keys), items ptr[v] .. ptr[v+1]-1 of perm have key v.  perm
// ([n]) and ptr ([nv+1]) are caller-owned device buffers; the scratch is stream-ordered.
int group_by_key_device(const int* keys, int n, int nv, int* perm, int* ptr, cudaStream_t st);

}  // namespace v3dba
