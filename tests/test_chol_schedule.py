"""The level schedule of the tile Cholesky (nested-dissection tile order, elimination-tree levels,
per-CTA task lists), checked on the CPU: the plan from v3dba_tile_schedule is executed here with
numpy exactly as k_chol_levels executes it (physical tile storage, transposed inputs, phase 1 /
phase 2 per level, back-substitution in reverse logical order) and must solve the system.

The reference orders the unknowns of its sparse LDL^T with block SYMAMD
(V3D/src/Math/v3d_optimization.cpp:54-98); any symmetric permutation gives the same solution, so
the check is against a dense solve (1e-12 relative: the 64x64 tiles are well conditioned)."""
import numpy as np
import pytest

from v3dsfmtoolkit_b200 import capi

TB = 64
FACTOR = 4   # task-mode flag of the phase-1 task that factors a diagonal tile


def band_arrow(nt, band=2):
    """Tile pattern of a sequence's reduced camera system: a band plus a dense last tile."""
    p = np.zeros((nt, nt), bool)
    for r in range(nt):
        for c in range(r + 1):
            p[r, c] = r - c <= band or r == nt - 1
    return p


def random_pattern(nt, density, seed):
    rng = np.random.default_rng(seed)
    p = np.tril(rng.random((nt, nt)) < density)
    np.fill_diagonal(p, True)
    return p


def groups(nt, size, seed):
    """Clusters of tiles with a few links between them."""
    rng = np.random.default_rng(seed)
    p = np.zeros((nt, nt), bool)
    for r in range(nt):
        for c in range(r + 1):
            p[r, c] = r // size == c // size or rng.random() < 0.02
    return p


def spd_from_pattern(pat, seed, pad=5):
    """SPD matrix with the tile pattern (lower tiles), diagonally dominant; the last `pad`
    unknowns are padding (identity rows) as in the solver's storage."""
    nt = pat.shape[0]
    n_pad = nt * TB
    n = n_pad - pad
    rng = np.random.default_rng(seed)
    A = np.zeros((n_pad, n_pad))
    for r in range(nt):
        for c in range(r + 1):
            if pat[r, c]:
                A[r * TB:(r + 1) * TB, c * TB:(c + 1) * TB] = 0.05 * rng.normal(size=(TB, TB))
    A = np.tril(A, -1)
    A = A + A.T
    A[n:, :] = 0.0
    A[:, n:] = 0.0
    A += np.diag(np.abs(A).sum(1) + 1.0 + np.abs(rng.normal(size=n_pad)))
    A[n:, n:] = np.eye(pad)
    b = np.concatenate([rng.normal(size=n), np.zeros(pad)])
    return A, b


def emulate(pat, A, b, sched):
    """Runs the plan on the physical storage the kernel uses: S (ld = n_pad + 64 rows, rhs in row
    n_pad), tiles addressed as S[rows, cols]."""
    nt = pat.shape[0]
    n_pad = nt * TB
    S = np.zeros((n_pad + TB, n_pad))
    S[:n_pad] = np.tril(A)
    S[n_pad] = b
    P = sched["plan"]
    perm = P["perm"]
    RANKS = sched["ranks"]

    def tile(pr, pc):
        return S[pr * TB:(pr + 1) * TB, pc * TB:(pc + 1) * TB]

    Z = np.zeros((nt, TB, TB))
    written = set()
    for lv in range(sched["n_levels"]):
        for rank in range(RANKS):
            for e in range(P["p1ptr"][lv * RANKS + rank], P["p1ptr"][lv * RANKS + rank + 1]):
                t = P["p1"][e]
                r, j, mode = P["task_r"][t], P["task_c"][t], P["task_mode"][t] & 3
                pr, pc = perm[r], perm[j]
                a = tile(pr, pc).copy() if mode == 1 else tile(pc, pr).T.copy() if mode == 2 else np.zeros((TB, TB))
                for u in range(P["task_cptr"][t], P["task_cptr"][t + 1]):
                    pk = perm[P["ck"][u]]
                    a -= tile(pr, pk) @ tile(pc, pk).T
                if P["task_mode"][t] & FACTOR:
                    L = np.linalg.cholesky(np.tril(a) + np.tril(a, -1).T)
                    Z[j] = np.linalg.inv(L)
                else:
                    tile(pr, pc)[:] = a
        for rank in range(RANKS):
            for e in range(P["p2ptr"][lv * RANKS + rank], P["p2ptr"][lv * RANKS + rank + 1]):
                t = P["p2"][e]
                r, j = P["task_r"][t], P["task_c"][t]
                pr, pc = perm[r], perm[j]
                assert (r, j) not in written
                written.add((r, j))
                a = tile(pc, pr).T.copy() if P["task_mode"][t] == 2 else tile(pr, pc).copy()
                tile(pr, pc)[:] = a @ Z[j].T
    # a level reads only what the levels above it solved: each level computes from a snapshot
    # taken before it, and an unsolved column (NaN) poisons the result
    x = np.full(n_pad, np.nan)
    done = []
    for lv in range(sched["n_levels"] - 1, -1, -1):
        before = x.copy()
        for rank in range(RANKS):
            for k in P["bcol"][P["blptr"][lv * RANKS + rank]:P["blptr"][lv * RANKS + rank + 1]]:
                k0 = perm[k] * TB
                v = S[n_pad, k0:k0 + TB].copy()
                for p in range(P["bptr"][k], P["bptr"][k + 1]):
                    r0 = perm[P["brow"][p]] * TB
                    v -= S[r0:r0 + TB, k0:k0 + TB].T @ before[r0:r0 + TB]
                x[k0:k0 + TB] = Z[k].T @ v
                done.append(k)
    assert sorted(done) == list(range(nt))
    return x, written


PATTERNS = [
    ("band_arrow19", band_arrow(19)),
    ("band_arrow40", band_arrow(40, band=3)),
    ("band12", band_arrow(12, band=1) & ~np.eye(12, k=-11, dtype=bool)),
    ("random20", random_pattern(20, 0.15, 3)),
    ("random9", random_pattern(9, 0.4, 4)),
    ("groups24", groups(24, 6, 5)),
    ("dense6", np.tril(np.ones((6, 6), bool))),
    ("single", np.ones((1, 1), bool)),
]


@pytest.mark.parametrize("ranks", [8, 16])
@pytest.mark.parametrize("name,pat", PATTERNS, ids=[p[0] for p in PATTERNS])
def test_level_schedule_solves_the_system(name, pat, ranks, monkeypatch):
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "levels")
    s = capi.tile_schedule(pat, ranks=ranks)
    nt = pat.shape[0]
    assert sorted(s["order"].tolist()) == list(range(nt))
    A, b = spd_from_pattern(pat, seed=nt)
    x, written = emulate(pat, A, b, s)
    xr = np.linalg.solve(A, b)
    assert np.abs(x - xr).max() <= 1e-12 * np.abs(xr).max()
    # every off-diagonal tile of L's pattern and every rhs tile is formed exactly once, every
    # diagonal tile factored once
    P = s["plan"]
    assert len(written) == len(P["p2"])
    assert sum(1 for (r, _) in written if r == nt) == nt
    assert sorted(P["task_c"][t] for t in P["p1"] if P["task_mode"][t] & FACTOR) == list(range(nt))


@pytest.mark.parametrize("name,pat", PATTERNS, ids=[p[0] for p in PATTERNS])
def test_plan_is_deterministic_and_tasks_are_disjoint(name, pat, monkeypatch):
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "levels")
    s1, s2 = capi.tile_schedule(pat), capi.tile_schedule(pat)
    RANKS = s1["ranks"]
    assert np.array_equal(s1["order"], s2["order"])
    for f in capi.LEVEL_PLAN_FIELDS:
        assert np.array_equal(s1["plan"][f], s2["plan"][f])
    P = s1["plan"]
    for ph in ("p1", "p2"):
        ptr, ids = P[ph + "ptr"], P[ph]
        assert len(ptr) == s1["n_levels"] * RANKS + 1 and ptr[-1] == len(ids)
        assert len(set(ids.tolist())) == len(ids)      # a task is in one phase list once
    # the level of a column is where its diagonal tile is factored; phase 1 of level L applies
    # updates of columns of earlier levels only (formed by then) to tiles whose column is not yet
    # factored, each target tile in at most one task per phase; phase 2 of level L forms level L's
    # panels only
    lvl = {}
    for lv in range(s1["n_levels"]):
        for e in range(P["p1ptr"][lv * RANKS], P["p1ptr"][(lv + 1) * RANKS]):
            t = P["p1"][e]
            if P["task_mode"][t] & FACTOR:
                lvl[P["task_c"][t]] = lv
    for lv in range(s1["n_levels"]):
        for e in range(P["p1ptr"][lv * RANKS], P["p1ptr"][(lv + 1) * RANKS]):
            t = P["p1"][e]
            for u in range(P["task_cptr"][t], P["task_cptr"][t + 1]):
                assert lvl[P["ck"][u]] <= lv - 1
            assert lvl[P["task_c"][t]] >= lv
        targets = [(P["task_r"][P["p1"][e]], P["task_c"][P["p1"][e]])
                   for e in range(P["p1ptr"][lv * RANKS], P["p1ptr"][(lv + 1) * RANKS])]
        assert len(set(targets)) == len(targets)
        for e in range(P["p2ptr"][lv * RANKS], P["p2ptr"][(lv + 1) * RANKS]):
            t = P["p2"][e]
            assert lvl[P["task_c"][t]] == lv and P["task_cptr"][t + 1] == P["task_cptr"][t]


def test_sequence_pattern_is_cut_into_few_levels():
    s = capi.tile_schedule(band_arrow(19))
    assert s["uses_levels"]
    assert s["order"][-1] == 18                       # the dense (intrinsics) tile is last
    assert s["n_levels"] <= 8
    assert s["est_levels_us"] < 0.85 * s["est_steps_us"]


# Per-CTA costs (µs) of k_chol_levels on B200, from its per-level phase timestamps on the
# 200-camera sequence pattern: a tile update with its operand loads, an update of a diagonal tile
# (lower triangle, one operand tile), an update of the rhs row, the factor of a diagonal tile, the
# load + store of an updated tile, a cluster barrier, a panel product, an rhs-row solve.
MEASURED_US = dict(gemm=3.5, gdiag=2.8, gemv=2.0, factor=9.0, tile=1.5, barrier=0.8, panel=3.8, solve=1.8)


def replay_phases(s, nt, c=MEASURED_US):
    """Phase-1 and phase-2 durations of every level of a plan: the longest CTA's task costs plus
    the barrier that ends the phase."""
    P, R = s["plan"], s["ranks"]
    p1, p2 = [], []
    for lv in range(s["n_levels"]):
        loads1, loads2 = np.zeros(R), np.zeros(R)
        for r in range(R):
            for t in P["p1"][P["p1ptr"][lv * R + r]:P["p1ptr"][lv * R + r + 1]]:
                nk = P["task_cptr"][t + 1] - P["task_cptr"][t]
                row, col = P["task_r"][t], P["task_c"][t]
                if row == nt:
                    loads1[r] += c["gemv"] * nk
                elif row == col:
                    loads1[r] += c["tile"] + c["gdiag"] * nk + (c["factor"] if P["task_mode"][t] & FACTOR else 0.0)
                else:
                    loads1[r] += c["tile"] + c["gemm"] * nk
            for t in P["p2"][P["p2ptr"][lv * R + r]:P["p2ptr"][lv * R + r + 1]]:
                loads2[r] += c["solve"] if P["task_r"][t] == nt else c["panel"]
        p1.append(loads1.max() + c["barrier"])
        p2.append(loads2.max() + c["barrier"])
    return np.array(p1), np.array(p2)


def test_sequence_plan_replayed_at_measured_costs():
    """The sequence plan replayed at the measured per-task costs: its phases sum to 169.2 µs, and
    the kernel's own timestamps for the same plan sum to 170.4 µs.  A planner that charged 3.5 µs
    per diagonal update and 1 µs per rhs update made a plan that replays at 183.7 µs; on the GPU
    the two plans took 0.2226 (that one) and 0.2135 ms (this one) per factor + solve."""
    s = capi.tile_schedule(band_arrow(19))
    p1, p2 = replay_phases(s, 19)
    assert p1.sum() + p2.sum() < 172.0
    assert p1.max() < 23.0                 # no phase longer than the top level's factor + 4 updates


def test_dense_pattern_keeps_the_column_kernel():
    s = capi.tile_schedule(np.tril(np.ones((12, 12), bool)))
    assert not s["uses_levels"]
    assert s["n_levels"] == 12


def test_schedule_can_be_forced(monkeypatch):
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "steps")
    s = capi.tile_schedule(band_arrow(19))
    assert not s["uses_levels"] and s["order"].tolist() == list(range(19))
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "levels")
    assert capi.tile_schedule(np.tril(np.ones((12, 12), bool)))["uses_levels"]


def test_invalid_arguments():
    with pytest.raises(capi.V3dbaError):
        capi.tile_schedule(np.zeros((0, 0), bool))
    for ranks in (1, 17):
        with pytest.raises(capi.V3dbaError):
            capi.tile_schedule(band_arrow(5), ranks=ranks)


def test_independent_and_arrow_patterns_have_one_and_two_levels(monkeypatch):
    monkeypatch.setenv("V3DBA_CHOL_SCHEDULE", "levels")
    diag = np.eye(20, dtype=bool)                        # no coupling: every column is a leaf
    s = capi.tile_schedule(diag)
    assert s["n_levels"] == 1
    arrow = np.eye(20, dtype=bool)
    arrow[19, :] = True                                 # one dense row (shared intrinsics alone)
    s = capi.tile_schedule(arrow)
    assert s["n_levels"] == 2 and s["order"][-1] == 19
    for pat in (diag, arrow):
        s = capi.tile_schedule(pat)
        A, b = spd_from_pattern(pat, seed=3)
        x, _ = emulate(pat, A, b, s)
        xr = np.linalg.solve(A, b)
        assert np.abs(x - xr).max() <= 1e-12 * np.abs(xr).max()
