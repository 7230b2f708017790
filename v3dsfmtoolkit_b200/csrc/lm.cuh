// Internal interfaces of the B200 bundle adjuster (not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "v3dba.h"

namespace v3dba {

constexpr int kRigStride = 24;   // doubles per rig camera: K 9, R 9, T 3, padding

struct ParamSet {
  double* K = nullptr;     // STD/VARYING: N*9, COMMON: 9
  double* R = nullptr;     // N*9
  double* T = nullptr;     // N*3
  double* dist = nullptr;  // COMMON: 4, VARYING: N*4, STD: 4 (unused)
  double* X = nullptr;     // M*3
};

struct Dims {
  int N = 0, M = 0, K = 0;
  int DA = 6, DC = 0;
  int model = 0, mode = 0;
  int nnA = 0, nnB = 0, nnC = 0;
  double thr = 1.0;
  double cached_ar = 1.0;
};

// Device-resident state of one problem.  Observations are in point-major order; each
// per-observation / per-point / per-camera block is stored contiguously with a padded stride
// (multiple of 16 bytes) so that it moves with vector loads.
struct DevState {
  Dims d;
  // structure
  int* o_cam = nullptr;     // [K] camera of permuted observation k
  int* o_pt = nullptr;      // [K] point of permuted observation k
  int* o_orig = nullptr;    // [K] caller's index of permuted observation k
  double* o_meas = nullptr; // [2K]
  int* p_ptr = nullptr;     // [M+1] track of point j = [p_ptr[j], p_ptr[j+1])
  int* p_order = nullptr;   // [M] points by descending track length, or null (large problems):
                            // k_linearize takes point p_order[t] in thread t, so a warp's
                            // tracks are equally long
  int* c_ptr = nullptr;     // [N+1]
  int* c_obs = nullptr;     // [K] permuted observation ids grouped by camera
  int* o_sub = nullptr;     // [K] rig camera of permuted observation k (STEREO)
  double* rig = nullptr;    // [n_rig][kRigStride] rig cameras K (9), R (9), T (3) (STEREO)
  int nb = 0;               // camera-pair blocks (i <= l) with at least one shared point
  int* b_i = nullptr;
  int* b_l = nullptr;
  int* b_ptr = nullptr;     // [nb+1] into the pair list
  int64_t P = 0;            // observation pairs
  int* pr_k = nullptr;      // [P] observation in camera b_i
  int* pr_m = nullptr;      // [P] observation in camera b_l
  // work chunks: camera observation lists cut into pieces of <= 64, pair lists into <= 128
  int nch_cam = 0;
  int* cc_beg = nullptr;    // [nch_cam] range in c_obs
  int* cc_end = nullptr;
  int* cam_cc_ptr = nullptr;  // [N+1] chunks of camera i
  int nch_blk = 0;
  int* bc_beg = nullptr;    // [nch_blk] range in the pair list
  int* bc_end = nullptr;
  int* blk_bc_ptr = nullptr;  // [nb+1] chunks of block b
  double* part_cc = nullptr;  // camera-chunk partials
  double* part_bc = nullptr;  // block-chunk partials
  // parameters
  ParamSet cur, trial, init;
  // per-observation (8-byte slots; FP32 mode uses the first half of each array)
  void* o_A = nullptr;      // 2*DA
  void* o_C = nullptr;      // 2*DC
  float* o_W = nullptr;     // DA*3   W_k = A_k^T B_k (FP32 blocks only)
  float* o_T = nullptr;     // DA*3   T_k = W_k Vinv_j (FP32 blocks only)
  double* o_B = nullptr;    // 2*3    B_k (FP64 blocks only; W and T are applied factor by factor)
  double* o_ga = nullptr;   // DA     A_k^T r_k (FP64)
  double* o_w = nullptr;    // Huber weights of the last linearisation
  // per point
  void* p_V = nullptr;      // 6 (upper triangle of B^T B)
  void* p_Y = nullptr;      // 3*DC
  void* p_Vinv = nullptr;   // 6
  void* p_YV = nullptr;     // 3*DC   Vinv Y
  double* p_gb = nullptr;   // 3
  double* p_q = nullptr;    // 3      Vinv gb
  // per camera
  void* c_U = nullptr;      // DA*DA
  void* c_X = nullptr;      // DA*DC
  double* c_ga = nullptr;   // DA
  // globals
  double* g_Z = nullptr;    // DC*DC
  double* g_gc = nullptr;   // DC
  // reduced system (dense, column-major, leading dimension ld)
  int n = 0, n_pad = 0, ld = 0;
  double* S = nullptr;
  double* rhs = nullptr;    // right-hand side, element c at rhs[c * rhs_stride]
  int rhs_stride = 0;       // ld for the dense system (row n_pad of S), 1 for PCG
  double* x = nullptr;      // [n_pad] solution of the reduced system
  void* Sb = nullptr;       // PCG: camera-pair blocks (Real, dA x dA row-major) instead of dense S
  int* diag_blk = nullptr;  // PCG: block id of (i, i)
  // scalars
  double* d_lambda = nullptr;
  double* d_relin = nullptr;  // {err, gmax, maxdiag}
  double* d_trial = nullptr;  // {new_err, d2, dg, failed}: d_relin + 4 (one readback for both)
  int* d_fail = nullptr;
  // reduction partials
  double* part = nullptr;
  size_t part_cap = 0;
  int relin_blocks_pt = 0, relin_blocks_cam = 0;
  int trial_blocks_pt = 0, trial_blocks_cam = 0, trial_blocks_obs = 0;
};

// Stages of one LM iteration, in launch order.
enum LmStage {
  kStageLinearize = 0,      // residuals, weights, Jacobian blocks, V/gb/Y per point, cost
  kStageCameraChunks = 1,   // partial U, ga, X per chunk of a camera's observations
  kStageCameraFinish = 2,   // U, ga, X per camera
  kStageRelinFinalize = 3,  // Z, gc, gradient max, max diagonal (initial lambda)
  kStagePointEliminate = 4, // (V + lambda I)^-1, T_k = W_k Vinv
  kStageSchurChunks = 5,    // partial camera-pair blocks per chunk of pairs
  kStageSchurFinish = 6,    // camera-pair blocks of S
  kStageRhsChunks = 7,      // partial reduced rhs / border per chunk
  kStageRhsFinish = 8,      // reduced rhs and camera/global border
  kStageGlobalBlock = 9,    // global block of S
  kStagePointBacksub = 10,  // point updates
  kStageCameraUpdate = 11,  // camera (and global) updates
  kStageTrialCost = 12,     // cost of the trial parameters with frozen weights
  kStageTrialFinalize = 13, // {new cost, |delta|^2, delta . g}
  kNumLmStages = 14
};

// partial sizes (doubles) of the chunk kernels for the worst case dims (dA = 13 / dC = 7)
size_t camera_chunk_values(int DA, int DC);
size_t block_chunk_values(int DA);

// Kernel sequence of one LM iteration, dispatched on (model, DA, DC) and storage precision.
struct LmOps {
  // linearise at cur: weights, Jacobian blocks, gradient, U/V/W/X/Y/Z, cost; if init_lambda,
  // *d_lambda = tau * max diagonal
  int (*relinearize)(DevState&, bool init_lambda, double tau, cudaStream_t);
  // Schur complement of the point blocks at *d_lambda into S / rhs (dense)
  int (*build_reduced)(DevState&, cudaStream_t);
  // back-substitution, trial parameters and their cost with frozen weights -> d_trial
  int (*finish_trial)(DevState&, cudaStream_t);
  // cost with Huber weights recomputed at the given parameters -> out[0]
  int (*cost)(DevState&, const ParamSet&, double* d_out, cudaStream_t);
  // one stage by id (LmStage)
  int (*stage)(DevState&, int id, int init_lambda, double tau, cudaStream_t);
};

size_t partial_doubles(const DevState& s);

const LmOps* lm_ops(int model, int DA, int DC, bool fp64);

constexpr int kLvFieldsMax = 16;   // room for the fields of LevelPlanField

// Tile-sparse dense FP64 Cholesky of the reduced system.
struct TileChol {
  int n = 0, n_pad = 0, nt = 0, ld = 0;
  static constexpr int TB = 64;
  std::vector<int> h_panel_ptr, h_panel_rows;   // per step k: tiles r > k with L(r,k) != 0
  std::vector<int> h_upd_ptr, h_upd_r, h_upd_c; // per step k: trailing tiles (r,c), k < c <= r
  std::vector<int> h_tiles;                     // every tile of L's pattern: r*nt + c
  int* d_panel_rows = nullptr;
  int* d_upd_r = nullptr;
  int* d_upd_c = nullptr;
  int* d_tiles = nullptr;
  int* d_panel_ptr = nullptr;
  int* d_upd_ptr = nullptr;
  double* d_ldiag = nullptr;                    // nt inverted diagonal tiles (L_kk^-1)
  // Level schedule under a nested-dissection order of the tiles (chol_order.cu).  When it
  // shortens the chain of dependent diagonal factorisations enough, tile_chol_solve runs
  // k_chol_levels with it instead of the column-by-column cluster kernel.
  bool levels = false;
  int n_levels = 0;
  int lv_ranks = 8;                             // CTAs of the cluster the plan was made for
  std::vector<int> h_order;                     // logical tile -> physical tile (nt + 1 entries)
  std::vector<int> h_lv;                        // the packed plan (offsets in lv_off)
  int lv_off[kLvFieldsMax] = {};
  int* d_lv = nullptr;
  double level_flops = 0.0;                     // algorithmic flops of the level schedule
  double est_levels_us = 0.0, est_steps_us = 0.0;  // the cost model's estimates of both kernels
};

constexpr int kLvFactor = 4;
// Offsets into TileChol::h_lv.
enum LevelPlanField {
  kLvP1Ptr = 0,   // [n_levels * ranks + 1] phase-1 task range of (level, cluster rank)
  kLvP1,          // phase-1 task ids (updates from the previous level, diagonal factors)
  kLvP2Ptr,       // [n_levels * ranks + 1] phase-2 task range of (level, cluster rank)
  kLvP2,          // phase-2 task ids (off-diagonal tiles and the rhs row)
  kLvTaskR,       // logical tile row of each task (nt: the rhs row)
  kLvTaskC,       // logical tile column of each task
  kLvTaskMode,    // where the input tile lives: 0 structurally zero, 1 S(pr, pc), 2 S(pc, pr)^T;
                  // | kLvFactor on the phase-1 task that factors a diagonal tile
  kLvTaskCPtr,    // [n_tasks + 1] updates of each task
  kLvCK,          // the column k of each update A_rc -= L_rk L_ck^T (phase-1 tasks)
  kLvPerm,        // [nt + 1] logical tile -> physical tile (entry nt: the rhs row)
  kLvBPtr,        // [nt + 1] back-substitution: rows r > k, r < nt, of L's logical column k
  kLvBRow,
  kLvBLvPtr,      // [n_levels * ranks + 1] back-substitution columns of (level, cluster rank)
  kLvBCol,
  kLvFields
};
// Orders the tiles (nested dissection of the tile graph, dense tiles last), builds the level
// schedule and decides whether tile_chol_solve uses it.  orig: the lower-triangle tile pattern
// before fill-in.
int tile_levels_plan(TileChol& tc, const std::vector<uint8_t>& orig);
// The host part of tile_levels_plan (no device work), for a cluster of `ranks` CTAs.
int tile_levels_build(TileChol& tc, const std::vector<uint8_t>& orig, int ranks);
// CTAs per cluster of k_chol_levels on this device: 16 where a 16-CTA cluster with its shared
// memory can be resident (a non-portable size, allowed on B200), else 8.
int chol_levels_ranks();
// The nested-dissection order alone (logical -> physical tile), for tests and the cost model.
std::vector<int> tile_nd_order(int nt, const std::vector<uint8_t>& orig);
int chol_levels_solve(const TileChol& tc, double* S, double* x, int* d_fail, cudaStream_t st,
                      unsigned long long* trace = nullptr);

// Block-sparse reduced system for block-Jacobi PCG.
struct PcgState {
  int* rp = nullptr;            // [N+1] camera rows over both triangles
  int* rb = nullptr;            // block id of each row entry
  int* rc = nullptr;            // column camera of each row entry
  unsigned char* rt = nullptr;  // 1: use the transpose of the stored block
  int* rd = nullptr;            // [N] entry of (i, i) in row i: the row's transposed entries
                                // (columns < i) come before it, its direct ones after it
  int* diag_blk = nullptr;      // [N] block id of (i, i)
  void* Sb = nullptr;           // blocks (8-byte slots)
  double* Pinv = nullptr;       // inverse diagonal blocks
  double* vec = nullptr;        // b, r, z, p, Ap
  double* b = nullptr;
  double* part = nullptr;
  double* gauge_rows = nullptr;  // [N x 28] per-camera terms of Z^T S Z
  double* gauge_L = nullptr;     // packed Cholesky factor of Z^T S Z and its ok flag
  int* iters = nullptr;
  bool ready = false;
};
int pcg_plan(PcgState& ps, const std::vector<int>& b_i, const std::vector<int>& b_l, int N);
int pcg_alloc(PcgState& ps, int nb, int N, int DA);
void pcg_free(PcgState& ps);
// Solves S x = b (b in ps.b, blocks in ps.Sb); iteration count in *ps.iters (device).
int pcg_solve(PcgState& ps, int N, int DA, bool fp64, double tol, int max_iter, double* x, int* d_fail,
              cudaStream_t st);

// Builds the plan from the lower-triangle tile pattern (tile_nz[r*nt+c], r >= c).
int tile_chol_plan(TileChol& tc, int n, std::vector<uint8_t>& tile_nz);
void tile_chol_free(TileChol& tc);
// Zeroes the pattern tiles of S (column-major, ld) and sets the padding diagonal to 1.
int tile_chol_zero(const TileChol& tc, double* S, double* rhs, cudaStream_t st);
// The same, and in the same launch the start of a trial: *d_lambda = lambda, *d_fail = 0.
int tile_chol_zero_setup(const TileChol& tc, double* S, double lambda, double* d_lambda, int* d_fail,
                         cudaStream_t st);
// Factors S in place and writes the solution to x; *d_fail = 1 on a non-positive pivot.
int tile_chol_solve(const TileChol& tc, double* S, double* x, int* d_fail, cudaStream_t st);
// Same factorisation and solve in one launch of an 8-CTA thread-block cluster.
int chol_cluster_solve(const TileChol& tc, double* S, double* x, int* d_fail, cudaStream_t st,
                       unsigned long long* trace = nullptr);
// The per-tile-column multi-launch variant (kept for very large reduced systems).
int tile_chol_solve_multilaunch(const TileChol& tc, double* S, double* x, int* d_fail, cudaStream_t st);

}  // namespace v3dba
