// Learned correction to the block-Jacobi preconditioner of the PCG reduced-camera solve, and the
// gauge coarse space (internal interface shared by precond_gnn.cu, pcg.cu and solver.cu).
#pragma once

#include <vector>

#include "common.cuh"
#include "lm.cuh"

namespace v3dba {

constexpr int kGnnH = 64;         // hidden width
constexpr int kGnnEdgeIn = 108;   // [F, (F F)|pattern, (F F^T)|pattern], three 6x6 blocks
constexpr int kGnnNodeIn = 4;     // [1, log(1 + degree), mean |F|^2, max |F|^2]
constexpr int kGnnOut = 3;        // c - 1 per edge
constexpr int kGnnProbes = V3DBA_PRECOND_PROBES;

// Weight layout: every linear layer is W (K x Nout, row-major) followed by its bias (Nout), so
// that [W; b] is one (K + 1) x Nout block.
struct GnnLayout {
  static constexpr int ein = 0;
  static constexpr int nin = ein + (kGnnEdgeIn + 1) * kGnnH;
  static constexpr int msz = (3 * kGnnH + 1) * kGnnH;
  static constexpr int m0 = nin + (kGnnNodeIn + 1) * kGnnH;
  static constexpr int hsz = (2 * kGnnH + 1) * kGnnH;
  static constexpr int h0 = m0 + 3 * msz;
  static constexpr int out = h0 + 2 * hsz;
  static constexpr int total = out + (kGnnH + 1) * kGnnOut;
};

// Camera co-visibility graph of a reduced system.  Edge e joins cameras a < b; it is the stored
// block (a, b) with id eblk[e], and stands for the lower position (b, a) of the factor.
struct GnnGraph {
  int N = 0, ne = 0, ntri = 0;
  int* ea = nullptr;
  int* eb = nullptr;
  int* eblk = nullptr;
  int* lo_ptr = nullptr;   // [N+1] edges (a, b) with b == node, ordered by a
  int* lo_e = nullptr;
  int* up_ptr = nullptr;   // [N+1] edges (a, b) with a == node, ordered by b
  int* up_e = nullptr;
  int* tri_ptr = nullptr;  // [ne+1] two-hop products of each edge
  int* tri_1 = nullptr;
  int* tri_2 = nullptr;
  unsigned char* tri_t = nullptr;   // 0: F(e1) F(e2); 1: F(e1) F(e2)^T
};

int gnn_graph_build(GnnGraph& g, int N, const std::vector<int>& b_i, const std::vector<int>& b_l);
void gnn_graph_free(GnnGraph& g);

// Normalised inputs of one system: cinv [N x 36], xe [ne x 108], xn [N x 4].  Sb holds the
// damped blocks (float when !fp64).  *d_fail = 1 when a diagonal block is not positive definite.
int gnn_features(const GnnGraph& g, const void* Sb, bool fp64, const int* diag_blk, float* cinv, float* xe,
                 float* xn, int* d_fail, cudaStream_t st);

// The PCG preconditioner blocks of the learned model for one system: ehat[blk] = E_e C_a^-1 for
// every edge (block-id indexed, 36 floats per block).  Runs the BF16 inference kernels.
int gnn_precond_blocks(v3dba_precond_model m, const GnnGraph& g, const float* cinv, const float* xe,
                       const float* xn, float* ehat, cudaStream_t st);

// Preconditioner of one PCG solve (pcg.cu): block-Jacobi unless the learned factor is given,
// plus the gauge coarse space when the camera frames are given.
struct PcgPrecond {
  const float* cinv = nullptr;     // [N x 36] lower-triangular C_i^-1
  const float* ehat = nullptr;     // [nb x 36] E_e C_a^-1 by block id
  const double* frames = nullptr;  // [N x 12] R_i (row-major) and T_i of every camera
};

int pcg_solve_precond(PcgState& ps, int N, int DA, bool fp64, double tol, int max_iter, double* x, int* d_fail,
                      cudaStream_t st, const PcgPrecond& P);

// Writes the gauge frames [N x 12] from the cameras' R (N x 9) and T (N x 3); the first
// n_fixed cameras (held fixed) get zero frames.
int gauge_frames(const double* R, const double* T, int N, int n_fixed, double* frames, cudaStream_t st);

}  // namespace v3dba
