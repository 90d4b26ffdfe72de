"""The reorder's CPU restatement (oracle.reorder_cm) and the tile count of the
reference's commit rule (oracle.tiles_8x4), on the CPU: the maps are
permutations, unreached rows / columns go last in index order, and the
traversal recovers a banded order from a scrambled one."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

import oracle as O
from rtt_spgemm import generators as G


def scrambled_band(n=400, half=6, seed=1):
    B = G.banded_scatter(n, half, scatter_max=0, seed=seed)
    p = np.random.default_rng(seed + 100).permutation(n)
    M = sp.csr_matrix((B.val, B.col, B.rowptr), shape=(n, n))[p][:, p].tocsr()
    M.sort_indices()
    return G.CSR(n, n, M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data)


def test_tiles_8x4_counts_distinct_tiles():
    A = G.CSR(9, 9, np.array([0, 2, 2, 2, 2, 2, 2, 2, 3, 4], np.int32),
              np.array([0, 5, 1, 8], np.int32), np.ones(4))
    # (row 0: cols 0, 5) -> tiles (0,0), (0,1); row 7 col 1 -> (0,0); row 8 col 8 -> (1,2)
    assert O.tiles_8x4(A) == 3
    # rows reversed: rows 8 and 1 land in different tile rows of 8 -> 4 tiles
    assert O.tiles_8x4(A, np.arange(9)[::-1], np.arange(9)) == 4


def test_reorder_cm_permutations_and_band_recovery():
    S = scrambled_band()
    r, c, comps, levels = O.reorder_cm(S)
    assert sorted(r) == list(range(S.m)) and sorted(c) == list(range(S.n))
    assert comps == 1 and levels > 10
    assert O.tiles_8x4(S, r, c) < O.tiles_8x4(S) // 3


def test_reorder_cm_empty_rows_last_and_components():
    # components {r0, c1}, {r1, c0}, {r3, r4, c3}; row 2 and columns 2, 4 empty
    A = G.CSR(5, 5, np.array([0, 1, 2, 2, 3, 4], np.int32), np.array([1, 0, 3, 3], np.int32),
              np.ones(4))
    r, c, comps, levels = O.reorder_cm(A)
    assert comps == 3
    assert r[2] == 4            # the empty row goes last
    assert c[2] == 3 and c[4] == 4  # unreached columns last, in index order


def _window_tiles(A, r, c, rows, W):
    """8x4 tiles of A per fine-pass window of the given axis."""
    ent_r = np.repeat(np.arange(A.m), np.diff(A.rowptr))
    R, Cc = np.asarray(r)[ent_r], np.asarray(c)[A.col]
    pos, grp, opp = (R, 8, Cc // 4) if rows else (Cc, 4, R // 8)
    keys = set(zip((pos // W).tolist(), ((pos % W) // grp).tolist(), opp.tolist()))
    out = {}
    for w, _, _ in keys:
        out[w] = out.get(w, 0) + 1
    return out


def test_fine_passes_are_monotone_per_window():
    """The fine passes' restatement: each pass gives permutations, moves
    indices only inside their window, and no window ends with more 8x4 tiles
    than it had; on a row-scrambled band (columns in order) the row pass
    removes tiles."""
    n = 256
    B = G.banded_scatter(n, 3, scatter_max=0, seed=3)
    p = np.random.default_rng(5).permutation(n)
    M = sp.csr_matrix((B.val, B.col, B.rowptr), shape=(n, n))[p].tocsr()
    M.sort_indices()
    A = G.CSR(n, n, M.indptr.astype(np.int32), M.indices.astype(np.int32), M.data)
    ident = np.arange(n)
    for rows, W in ((True, 32), (False, 16)):
        r, c, st = O.reorder_fine_pass(A, ident, ident, rows)
        moved = r if rows else c
        assert sorted(moved) == list(range(n))
        assert np.array_equal(moved // W, ident // W)  # inside the windows
        before, after = _window_tiles(A, ident, ident, rows, W), _window_tiles(A, r, c, rows, W)
        assert all(after.get(w, 0) <= t for w, t in before.items())
        assert st["windows"] == (n + W - 1) // W
        assert O.tiles_8x4(A, r, c) == O.tiles_8x4(A) - st["reduction"]
    r, c, st = O.reorder_fine_pass(A, ident, ident, True)
    assert st["reduction"] > 0 and st["accepted"] > 0


def test_reorder_plan_variants_never_add_tiles():
    S = scrambled_band(300, 5, seed=7)
    for variant in range(5):
        r, c, info = O.reorder_plan(S, variant)
        assert sorted(r) == list(range(S.m)) and sorted(c) == list(range(S.n))
        assert info["tiles_after"] <= info["tiles_before"], variant
    # the full plan: the coarse stage, then the fine passes on top of it
    r, c, info = O.reorder_plan(S, 0)
    assert info["accepted"] == 1
    assert info["tiles_after"] == info["proposal_tiles"] - info["row"]["reduction"] - \
        info["inner"]["reduction"]
