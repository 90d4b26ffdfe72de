"""GPU: the diagnostics of the tile layout - the reorder plan dump in the
reference's three-file format (dump_dmma_reorder_plan,
src/dmma_reorder.h:3087) and the tile heatmaps of A, B and C (the role of
export_diagnostic_heatmaps, src/super16_symbolic.cuh:2034) - against the
plan's maps and the oracle's tiles."""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev(A):
    d = torch.device("cuda:0")
    return (A.m, A.n, torch.from_numpy(A.rowptr).to(d), torch.from_numpy(A.col).to(d),
            torch.from_numpy(A.val).to(d))


def test_reorder_plan_dump(tmp_path):
    A = G.stencil_27(6, 2).permute_symmetric(np.random.default_rng(3).permutation(216))
    ctx = R.Context(0)
    stem = tmp_path / "plan"
    plan = ctx.reorder_plan_dump(_dev(A), str(stem))
    rows = [l.split(",") for l in (tmp_path / "plan_permutations.csv").read_text().splitlines()]
    assert rows[0] == ["axis", "old_id", "new_id", "new_to_old_at_new_id"]
    body = rows[1:]
    assert len(body) == A.m + A.n
    for axis, o, nw, back in body:
        assert back == o  # new_to_old[old_to_new[old]] == old
        key = "row_old_to_new" if axis == "row" else "inner_old_to_new"
        assert plan[key][int(o)] == int(nw)
    stats = dict(l.split(",") for l in
                 (tmp_path / "plan_unified_stats.csv").read_text().splitlines()[1:])
    assert int(stats["tiles_before"]) == plan["tiles_before"]
    assert int(stats["tiles_after"]) == plan["tiles_after"] <= plan["tiles_before"]
    M = R.mmio_read(tmp_path / "plan_A_reordered.mtx")
    assert (M.m, M.n, M.nnz) == (A.m, A.n, A.nnz)
    rows_old = np.repeat(np.arange(A.m), np.diff(A.rowptr))
    want = set(zip(plan["row_old_to_new"][rows_old].tolist(),
                   plan["inner_old_to_new"][A.col].tolist()))
    got = set(zip(np.repeat(np.arange(M.m), np.diff(M.rowptr)).tolist(), M.col.tolist()))
    assert got == want
    ctx.close()


@pytest.mark.parametrize("bins", [1, 7, 64])
def test_tile_heatmaps(orc, bins):
    A = G.banded_scatter(900, 20, seed=11)
    ctx = R.Context(0)
    da = _dev(A)
    nnz, tiles = ctx.symbolic(da)
    ta = orc.csr2tile_row_major(A)
    tm, tn = ta["tilem"], ta["tilen"]
    I = np.repeat(np.arange(tm), np.diff(ta["tile_ptr"]))
    J = ta["tile_columnidx"]
    # C's tiles: the tile-level product of A's tile pattern with B's (= A's),
    # as step 1 forms it (a tile whose entries all cancel structurally stays)
    TA = np.zeros((tm, tn), bool)
    TA[I, J] = True
    TC = (TA.astype(np.int64) @ TA.astype(np.int64)) > 0
    CI, CJ = np.nonzero(TC)
    for which, (ii, jj) in (("A", (I, J)), ("B", (I, J)), ("C", (CI, CJ))):
        h = ctx.tile_heatmap(which, bins)
        want = np.zeros((bins, bins), np.uint64)
        np.add.at(want, (ii * bins // tm, jj * bins // tn), 1)
        assert np.array_equal(h, want), which
    assert int(ctx.tile_heatmap("C", bins).sum()) == tiles
    ctx.close()
