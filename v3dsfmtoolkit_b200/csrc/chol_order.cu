// Tile ordering and level schedule of the reduced-system Cholesky (host side).
//
// The column-by-column cluster kernel (chol_cluster.cu) factors the diagonal tiles one after
// another: its time is nt x (one 64x64 factor + two tile GEMMs) whatever the sparsity.  The
// reduced camera system of a sequence is a band of tiles plus the dense intrinsics tile, whose
// elimination tree in the natural order is a chain.  Here the tiles are renumbered by nested
// dissection of the tile graph (George's level-structure bisection, applied recursively; tiles
// adjacent to at least half of the others, such as the intrinsics tile, are numbered last), the
// fill-in and the elimination tree of the renumbered pattern are found, and every tile column is
// given a level = its height in that tree.  Columns of one level are independent: the cluster
// kernel k_chol_levels factors them concurrently, with one cluster barrier per phase.
//
// The order is a symmetric permutation of whole 64x64 tiles: the factor of P S P^T solves the
// same system, and the solution is written back in the caller's order.  Nothing is copied: a
// logical tile (r, c), r >= c, lives at the physical tile (perm r, perm c) of S, which is in the
// upper triangle when perm r < perm c (storage the assembly never uses); its input is then the
// transpose of the assembled lower tile (perm c, perm r).
//
// This replaces the reference's fill-reducing ordering of the sparse LDL^T (block SYMAMD,
// V3D/src/Math/v3d_optimization.cpp:54-98): both renumber the camera unknowns before the
// factorisation; this one minimises the height of the elimination tree (the critical path on a
// parallel machine) rather than the fill.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iterator>
#include <map>
#include <vector>

#include "common.cuh"
#include "lm.cuh"

namespace v3dba {

namespace {

// cost model of one CTA, in microseconds: a 64x64x64 DMMA tile product with its operand loads,
// the factor + inverse of one diagonal tile, a cluster barrier, and the store of an updated tile
constexpr double kGemmUs = 2.0, kFactorUs = 20.0, kBarrierUs = 1.0, kStoreUs = 0.5;
// the same for one update or solve of the rhs row (a GEMV over one tile)
constexpr double kGemvUs = 0.6;
// Measured on B200 (sequence200 pattern, per CTA): one tile update with its operand loads, one
// update of a diagonal tile (its lower triangle only, one operand tile), the factor of a diagonal
// tile, the load + store of an updated tile, one update of the rhs row.  They size the phase
// budget into which updates that are not yet due are moved.  (A sweep of the update / factor
// costs over 3.5-6 / 9-14 us moved the sequence200 factor + solve between 0.234 and 0.252 ms;
// applying every update only when due took 0.334 ms.  The diagonal-update and rhs costs are
// fitted to the phase times of the kernel's own timestamps.)
constexpr double kMeasGemmUs = 3.5, kMeasDiagUs = 2.8, kMeasFactorUs = 9.0, kMeasTileUs = 1.5, kMeasGemvUs = 2.0;

struct TileGraph {
  int nt = 0;
  std::vector<std::vector<int>> adj;
};

// Breadth-first levels from s over the vertices with in_set[v] == tag.
void bfs_levels(const TileGraph& g, const std::vector<int>& in_set, int tag, int s, std::vector<int>& lev,
                std::vector<int>& order) {
  order.clear();
  lev[s] = 0;
  order.push_back(s);
  for (size_t h = 0; h < order.size(); ++h) {
    const int u = order[h];
    for (int w : g.adj[u])
      if (in_set[w] == tag && lev[w] < 0) {
        lev[w] = lev[u] + 1;
        order.push_back(w);
      }
  }
}

// Appends the nested-dissection order of the vertex set V (in_set[v] == tag) to out.
void nd_order(const TileGraph& g, std::vector<int> V, std::vector<int>& in_set, int& next_tag,
              std::vector<int>& out) {
  std::sort(V.begin(), V.end());
  if (V.size() <= 3) {
    out.insert(out.end(), V.begin(), V.end());
    return;
  }
  const int tag = next_tag++;
  for (int v : V) in_set[v] = tag;
  std::vector<int> lev(g.nt, -1), order;
  // connected components: each is an independent subtree
  std::vector<std::vector<int>> comps;
  for (int s : V)
    if (lev[s] < 0) {
      bfs_levels(g, in_set, tag, s, lev, order);
      comps.push_back(order);
    }
  if (comps.size() > 1) {
    for (auto& c : comps) nd_order(g, c, in_set, next_tag, out);
    return;
  }
  // pseudo-peripheral start: repeat BFS from the (lowest-numbered) farthest vertex
  int s = V[0];
  for (int it = 0; it < 4; ++it) {
    for (int v : V) lev[v] = -1;
    bfs_levels(g, in_set, tag, s, lev, order);
    int far = 0;
    for (int v : V) far = std::max(far, lev[v]);
    int t = g.nt;
    for (int v : V)
      if (lev[v] == far) t = std::min(t, v);
    if (t == s) break;
    s = t;
  }
  for (int v : V) lev[v] = -1;
  bfs_levels(g, in_set, tag, s, lev, order);
  int far = 0;
  for (int v : V) far = std::max(far, lev[v]);
  if (far < 2) {
    out.insert(out.end(), V.begin(), V.end());
    return;
  }
  // separator: the level at which half of the vertices have been reached
  std::vector<int> cnt(far + 1, 0);
  for (int v : V) cnt[lev[v]]++;
  int m = 0, acc = 0;
  for (; m <= far; ++m) {
    acc += cnt[m];
    if (2 * acc >= (int)V.size()) break;
  }
  m = std::max(1, std::min(m, far - 1));
  std::vector<int> A, B, S;
  for (int v : V) (lev[v] < m ? A : lev[v] > m ? B : S).push_back(v);
  nd_order(g, A, in_set, next_tag, out);
  nd_order(g, B, in_set, next_tag, out);
  out.insert(out.end(), S.begin(), S.end());
}

// Greedy longest-processing-time assignment of tasks (cost) to the cluster's `ranks` CTAs; ties
// go to the lowest rank and equal costs keep their order, so the schedule is deterministic.
std::vector<std::vector<int>> assign_lpt(const std::vector<int>& tasks, const std::vector<double>& cost, int ranks,
                                         double* makespan) {
  std::vector<int> idx(tasks.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<std::vector<int>> per(ranks);
  std::vector<double> load(ranks, 0.0);
  for (int i : idx) {
    int best = 0;
    for (int r = 1; r < ranks; ++r)
      if (load[r] < load[best]) best = r;
    load[best] += cost[i];
    per[best].push_back(tasks[i]);
  }
  *makespan = *std::max_element(load.begin(), load.end());
  return per;
}

}  // namespace

std::vector<int> tile_nd_order(int nt, const std::vector<uint8_t>& orig) {
  TileGraph g;
  g.nt = nt;
  g.adj.assign(nt, {});
  for (int r = 0; r < nt; ++r)
    for (int c = 0; c < r; ++c)
      if (orig[(size_t)r * nt + c]) {
        g.adj[r].push_back(c);
        g.adj[c].push_back(r);
      }
  // dense tiles (adjacent to at least half of the others) are numbered last, in their order
  std::vector<int> rest, dense;
  const int dense_deg = std::max(4, (nt - 1 + 1) / 2);
  for (int v = 0; v < nt; ++v) ((int)g.adj[v].size() >= dense_deg ? dense : rest).push_back(v);
  std::vector<int> in_set(nt, -1), out;
  int next_tag = 0;
  nd_order(g, rest, in_set, next_tag, out);
  out.insert(out.end(), dense.begin(), dense.end());
  return out;
}

int tile_levels_build(TileChol& tc, const std::vector<uint8_t>& orig, int ranks) {
  const int nt = tc.nt;
  if (ranks < 2) return V3DBA_ERR_INVALID_ARGUMENT;
  tc.lv_ranks = ranks;
  tc.levels = false;
  tc.h_lv.clear();
  tc.h_order.clear();
  const char* force = std::getenv("V3DBA_CHOL_SCHEDULE");
  const bool force_levels = force && std::strcmp(force, "levels") == 0;
  const bool force_steps = force && std::strcmp(force, "steps") == 0;
  if (force_steps || nt < 1) return V3DBA_OK;

  std::vector<int> perm = tile_nd_order(nt, orig);
  // logical pattern with fill-in
  std::vector<uint8_t> L((size_t)nt * nt, 0);
  auto O = [&](int pr, int pc) { return pr == pc || orig[(size_t)std::max(pr, pc) * nt + std::min(pr, pc)] != 0; };
  for (int r = 0; r < nt; ++r)
    for (int c = 0; c <= r; ++c)
      if (O(perm[r], perm[c])) L[(size_t)r * nt + c] = 1;
  std::vector<std::vector<int>> colrows(nt);   // rows r > k of column k (ascending)
  for (int k = 0; k < nt; ++k) {
    for (int r = k + 1; r < nt; ++r)
      if (L[(size_t)r * nt + k]) colrows[k].push_back(r);
    const auto& rows = colrows[k];
    for (size_t a = 0; a < rows.size(); ++a)
      for (size_t b = 0; b <= a; ++b) L[(size_t)rows[a] * nt + rows[b]] = 1;
  }
  // elimination tree heights
  std::vector<int> level(nt, 0);
  int n_levels = 0;
  for (int k = 0; k < nt; ++k) {
    if (!colrows[k].empty()) level[colrows[k][0]] = std::max(level[colrows[k][0]], level[k] + 1);
    n_levels = std::max(n_levels, level[k] + 1);
  }
  // Tasks.  An update A_ab -= L_ak L_bk^T (rows a >= b of column k, and the rhs row) can run in
  // phase 1 of any level after column k's panels are formed (the phase 2 of level[k]) and must
  // have run by phase 1 of level[b], where tile (a, b) is factored (a == b) or consumed by the
  // panel product of phase 2 (a > b).  Phase 1 of level L takes, as one task per target tile
  // (its columns k ascending), every pending update that is due at L, and factors the diagonal
  // tiles of level L once their last updates are in; the CTAs are loaded by longest processing
  // time first.  Updates not yet due then fill the CTAs up to that phase's longest load (earliest
  // due first), and what does not fit waits for a later phase: the phase lasts no longer, and the
  // later, narrower levels take work off the wide early ones.  Phase 2 of level L forms
  // L_rj = A_rj Z_j^T for the off-diagonal tiles of level L's columns.  A tile is read as
  // assembled (mode 0/1/2) the first time it is touched and in place (mode 1) after that;
  // kLvFactor marks the diagonal tasks that factor.
  std::vector<int> t_r, t_c, t_mode, t_cptr(1, 0), c_k;
  std::vector<std::vector<int>> lv_cols(n_levels);
  for (int j = 0; j < nt; ++j) lv_cols[level[j]].push_back(j);
  std::vector<uint8_t> touched((size_t)(nt + 1) * nt, 0);
  auto input_mode = [&](int r, int c) -> int {
    if (r == c || r == nt || touched[(size_t)r * nt + c]) return 1;
    const int pr = perm[r], pc = perm[c];
    return O(pr, pc) ? (pr > pc ? 1 : 2) : 0;
  };
  std::vector<int> p1ptr(1, 0), p1, p2ptr(1, 0), p2;
  bool consistent = true;
  double est = 0.0, flops = 0.0;
  const double gemm = 2.0 * 64.0 * 64.0 * 64.0;
  auto make_task = [&](int r, int c, const int* ks, int nk, bool factor) {
    const int id = (int)t_r.size();
    t_r.push_back(r);
    t_c.push_back(c);
    t_mode.push_back(input_mode(r, c) | (factor ? kLvFactor : 0));
    touched[(size_t)r * nt + c] = 1;
    for (int u = 0; u < nk; ++u) c_k.push_back(ks[u]);
    t_cptr.push_back((int)c_k.size());
    flops += (r == nt ? 2.0 * 64.0 * 64.0 : gemm) * nk + (factor ? 64.0 * 64.0 * 64.0 : 0.0);
    return id;
  };
  std::map<std::pair<int, int>, std::vector<int>> pending;   // target (r, c) -> columns k not yet applied
  for (int lv = 0; lv < n_levels; ++lv) {
    if (lv > 0)
      for (int k : lv_cols[lv - 1]) {
        std::vector<int> rows = colrows[k];
        rows.push_back(nt);
        for (size_t a = 0; a < rows.size(); ++a)
          for (size_t b = 0; b <= a; ++b)
            if (rows[b] < nt) pending[{rows[a], rows[b]}].push_back(k);
      }
    for (int j : lv_cols[lv]) pending[{j, j}];
    // the updates due at this level, one task per target
    std::vector<int> ph1, ph2;
    std::vector<double> cost1, meas1, cost2;
    for (auto it = pending.begin(); it != pending.end();) {
      const int r = it->first.first, c = it->first.second;
      if (level[c] != lv) {
        ++it;
        continue;
      }
      const bool factor = r == c;
      const int nc = (int)it->second.size();
      if (!factor && nc == 0) {   // all of its updates ran early
        it = pending.erase(it);
        continue;
      }
      ph1.push_back(make_task(r, c, it->second.data(), nc, factor));
      cost1.push_back(factor ? kFactorUs + kGemmUs * nc : (r == nt ? kGemvUs : kGemmUs) * nc + kStoreUs);
      meas1.push_back(factor ? kMeasFactorUs + kMeasTileUs + kMeasDiagUs * nc
                             : r == nt ? kMeasGemvUs * nc : kMeasGemmUs * nc + kMeasTileUs);
      it = pending.erase(it);
    }
    double m1 = 0.0, m2 = 0.0, mm = 0.0;
    auto a1 = assign_lpt(ph1, cost1, ranks, &m1);
    std::vector<double> load(ranks, 0.0);
    {   // the loads of that assignment under the measured costs
      std::vector<int> pos(t_r.size(), -1);
      for (size_t i = 0; i < ph1.size(); ++i) pos[ph1[i]] = (int)i;
      for (int r = 0; r < ranks; ++r)
        for (int id : a1[r]) load[r] += meas1[pos[id]];
      mm = *std::max_element(load.begin(), load.end());
    }
    // updates not yet due, earliest due first (then the target's order), into the slack below
    // the phase's longest load
    std::vector<std::pair<int, int>> opt;
    for (auto& pd : pending)
      if (!pd.second.empty()) opt.push_back(pd.first);
    std::stable_sort(opt.begin(), opt.end(), [&](const std::pair<int, int>& x, const std::pair<int, int>& y) {
      return level[x.second] < level[y.second];
    });
    for (const auto& key : opt) {
      std::vector<int>& ks = pending[key];
      const int r = key.first, c = key.second;
      const double g = r == nt ? kMeasGemvUs : (r == c ? kMeasDiagUs : kMeasGemmUs), fixed = r == nt ? 0.0 : kMeasTileUs;
      int best = 0;
      for (int q = 1; q < ranks; ++q)
        if (load[q] < load[best]) best = q;
      const int fit = (int)std::min<double>((double)ks.size(), std::floor((mm - load[best] - fixed) / g + 1e-9));
      if (fit < 1) continue;
      const int id = make_task(r, c, ks.data(), fit, false);
      a1[best].push_back(id);
      load[best] += fixed + g * fit;
      ks.erase(ks.begin(), ks.begin() + fit);
    }
    for (auto it = pending.begin(); it != pending.end();) it = it->second.empty() ? pending.erase(it) : std::next(it);
    for (int j : lv_cols[lv]) {
      std::vector<int> rows = colrows[j];
      rows.push_back(nt);
      for (int r : rows) {
        const int id = (int)t_r.size();
        const int mode = input_mode(r, j);
        if (mode == 0) consistent = false;   // a zero tile of L's pattern that no update reached
        t_r.push_back(r);
        t_c.push_back(j);
        t_mode.push_back(mode);
        touched[(size_t)r * nt + j] = 1;
        t_cptr.push_back((int)c_k.size());
        flops += r == nt ? 2.0 * 64.0 * 64.0 : gemm;
        ph2.push_back(id);
        cost2.push_back(r == nt ? kGemvUs : kGemmUs);
      }
    }
    auto a2 = assign_lpt(ph2, cost2, ranks, &m2);
    for (int r = 0; r < ranks; ++r) {
      p1.insert(p1.end(), a1[r].begin(), a1[r].end());
      p1ptr.push_back((int)p1.size());
      p2.insert(p2.end(), a2[r].begin(), a2[r].end());
      p2ptr.push_back((int)p2.size());
    }
    est += m1 + m2 + 2.0 * kBarrierUs;
  }
  for (const auto& pd : pending)
    if (!pd.second.empty()) consistent = false;   // an update that was never due (cannot happen)
  std::vector<int> bptr(1, 0), brow;
  for (int k = 0; k < nt; ++k) {
    brow.insert(brow.end(), colrows[k].begin(), colrows[k].end());
    bptr.push_back((int)brow.size());
  }
  // back-substitution: the columns of a level are independent once their ancestors (higher
  // levels) are solved; column i of a level goes to rank i mod ranks
  std::vector<int> blptr(1, 0), bcol;
  for (int lv = 0; lv < n_levels; ++lv)
    for (int r = 0; r < ranks; ++r) {
      for (size_t i = r; i < lv_cols[lv].size(); i += ranks) bcol.push_back(lv_cols[lv][i]);
      blptr.push_back((int)bcol.size());
    }
  perm.push_back(nt);

  tc.n_levels = n_levels;
  tc.level_flops = flops;
  tc.est_levels_us = est;
  tc.est_steps_us = nt * (kFactorUs + 3.0 * kGemmUs + 2.0 * kBarrierUs);
  tc.h_order = perm;
  static_assert(kLvFields <= kLvFieldsMax, "level plan fields");
  const std::vector<int>* parts[kLvFields] = {&p1ptr, &p1, &p2ptr, &p2, &t_r, &t_c, &t_mode, &t_cptr,
                                              &c_k, &perm, &bptr, &brow, &blptr, &bcol};
  for (int f = 0; f < kLvFields; ++f) {
    tc.lv_off[f] = (int)tc.h_lv.size();
    tc.h_lv.insert(tc.h_lv.end(), parts[f]->begin(), parts[f]->end());
  }
  tc.levels = consistent && (force_levels || (nt >= 4 && est < 0.85 * tc.est_steps_us));
  return V3DBA_OK;
}

int tile_levels_plan(TileChol& tc, const std::vector<uint8_t>& orig) {
  if (tc.d_lv) {
    cudaFree(tc.d_lv);
    tc.d_lv = nullptr;
  }
  const int rc = tile_levels_build(tc, orig, chol_levels_ranks());
  if (rc || !tc.levels) return rc;
  if (injected_alloc_failure()) return V3DBA_ERR_OUT_OF_MEMORY;
  V3DBA_CUDA_TRY(cudaMalloc(&tc.d_lv, sizeof(int) * std::max<size_t>(tc.h_lv.size(), 1)));
  V3DBA_CUDA_TRY(cudaMemcpy(tc.d_lv, tc.h_lv.data(), sizeof(int) * tc.h_lv.size(), cudaMemcpyHostToDevice));
  return V3DBA_OK;
}

}  // namespace v3dba

extern "C" int v3dba_tile_schedule(int nt, const uint8_t* pattern, int ranks, int* order, int* n_levels,
                                   int* uses_levels, double* est_us, int* plan, int plan_cap, int* plan_len,
                                   int* offsets) {
  if (nt <= 0 || !pattern || ranks < 2 || ranks > 16 || !order || !n_levels || !uses_levels || !est_us ||
      !plan_len || !offsets)
    return V3DBA_ERR_INVALID_ARGUMENT;
  v3dba::TileChol tc;
  tc.nt = nt;
  tc.n_pad = nt * v3dba::TileChol::TB;
  tc.n = tc.n_pad;
  tc.ld = tc.n_pad + v3dba::TileChol::TB;
  std::vector<uint8_t> orig(pattern, pattern + (size_t)nt * nt);
  for (int k = 0; k < nt; ++k) orig[(size_t)k * nt + k] = 1;
  const int rc = v3dba::tile_levels_build(tc, orig, ranks);
  if (rc) return rc;
  if (tc.h_order.empty()) {   // the column-by-column schedule was forced: natural order
    for (int k = 0; k < nt; ++k) order[k] = k;
    *n_levels = nt;
    *uses_levels = 0;
    est_us[0] = est_us[1] = 0.0;
    *plan_len = 0;
    return V3DBA_OK;
  }
  for (int k = 0; k < nt; ++k) order[k] = tc.h_order[k];
  *n_levels = tc.n_levels;
  *uses_levels = tc.levels ? 1 : 0;
  est_us[0] = tc.est_levels_us;
  est_us[1] = tc.est_steps_us;
  *plan_len = (int)tc.h_lv.size();
  for (int f = 0; f < v3dba::kLvFields; ++f) offsets[f] = tc.lv_off[f];
  if (plan && plan_cap >= (int)tc.h_lv.size()) std::copy(tc.h_lv.begin(), tc.h_lv.end(), plan);
  return V3DBA_OK;
}
