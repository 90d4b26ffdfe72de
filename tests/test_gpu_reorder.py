"""GPU parity of the reorder (rtt_reorder_plan_build, the reference's
build_dmma_reorder_plan: coarse traversal under the exact commit rule, then
the row and inner fine passes) and of rtt_csr_permute: the maps and counters
of every variant equal the CPU restatement's, the tile counts equal the
oracle's, a guarded plan never has more 8x4 A tiles than A, and a product
through reordered operands gives the same C once its rows are restored."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
import rtt_spgemm as R
from rtt_spgemm import generators as G
from conftest import assert_csr_close
from test_reorder_cpu import scrambled_band

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
DEV = torch.device("cuda:0")


def _dev(A):
    return (A.m, A.n, torch.from_numpy(A.rowptr).to(DEV), torch.from_numpy(A.col).to(DEV),
            torch.from_numpy(A.val).to(DEV))


def _host(c):
    m, n, rp, ci, va = c
    return G.CSR(m, n, rp.cpu().numpy(), ci.cpu().numpy(), va.cpu().numpy())


CASES = {
    "scrambled_band": lambda: scrambled_band(),
    "scrambled_band_2k": lambda: scrambled_band(2000, 9, seed=4),
    "lap2d_40": lambda: G.laplacian_2d(40),
    "rmat_10": lambda: G.rmat(10, 8, seed=2),
    "rect_random": lambda: G.random_csr(300, 500, 0.01, seed=5),
    "components": lambda: G.CSR(5, 5, np.array([0, 1, 2, 2, 3, 4], np.int32),
                                np.array([1, 0, 3, 3], np.int32), np.ones(4)),
}


@pytest.mark.parametrize("case", list(CASES))
def test_reorder_plan_matches_restatement(case):
    """The coarse stage alone (RTT_REORDER_COARSE): the traversal's maps and
    the commit rule against the CPU restatement."""
    A = CASES[case]()
    ctx = R.Context(0)
    plan = ctx.reorder_plan(_dev(A), R.RTT_REORDER_COARSE)
    ctx.close()
    r, c, comps, levels = O.reorder_cm(A)
    assert plan["tiles_before"] == O.tiles_8x4(A)
    assert plan["proposal_tiles"] == O.tiles_8x4(A, r, c)
    assert (plan["components"], plan["levels"]) == (comps, levels)
    assert plan["accepted"] == int(plan["proposal_tiles"] < plan["tiles_before"])
    assert plan["tiles_after"] <= plan["tiles_before"]
    if plan["accepted"]:
        assert np.array_equal(plan["row_old_to_new"], r)
        assert np.array_equal(plan["inner_old_to_new"], c)
        assert plan["tiles_after"] == plan["proposal_tiles"]
    else:
        assert np.array_equal(plan["row_old_to_new"], np.arange(A.m))
        assert np.array_equal(plan["inner_old_to_new"], np.arange(A.n))
    assert np.array_equal(plan["row_new_to_old"][plan["row_old_to_new"]], np.arange(A.m))
    assert np.array_equal(plan["inner_new_to_old"][plan["inner_old_to_new"]], np.arange(A.n))


@pytest.mark.parametrize("variant", [R.RTT_REORDER_FULL, R.RTT_REORDER_FINE,
                                     R.RTT_REORDER_COARSE_ROW, R.RTT_REORDER_COARSE_INNER,
                                     R.RTT_REORDER_UNGUARDED])
@pytest.mark.parametrize("case", list(CASES))
def test_reorder_fine_passes_match_restatement(case, variant):
    """Every stage of every variant - the coarse traversal under the commit
    rule, the row pass (windows of 32, groups of 8) and the inner pass
    (windows of 16, groups of 4), each window committed by its exact tile
    count and fan-out - gives the maps and counters of the CPU restatement
    (oracle.reorder_plan), bit for bit."""
    A = CASES[case]()
    ctx = R.Context(0)
    plan = ctx.reorder_plan(_dev(A), variant)
    ctx.close()
    r, c, info = O.reorder_plan(A, variant)
    assert np.array_equal(plan["row_old_to_new"], r)
    assert np.array_equal(plan["inner_old_to_new"], c)
    assert np.array_equal(plan["row_new_to_old"][plan["row_old_to_new"]], np.arange(A.m))
    assert np.array_equal(plan["inner_new_to_old"][plan["inner_old_to_new"]], np.arange(A.n))
    assert plan["variant"] == variant
    assert plan["tiles_before"] == info["tiles_before"]
    assert plan["tiles_after"] == info["tiles_after"] == O.tiles_8x4(A, r, c)
    assert plan["accepted"] == info["accepted"]
    for axis in ("row", "inner"):
        if axis in info:
            st = info[axis]
            assert plan[f"{axis}_windows"] == st["windows"]
            assert plan[f"accepted_{axis}_windows"] == st["accepted"]
            assert plan[f"{axis}_tile_reduction"] == st["reduction"]
            assert plan[f"{axis}_fanout_before"] == st["fanout_before"]
            assert plan[f"{axis}_fanout_after"] == st["fanout_after"]
        else:
            assert plan[f"{axis}_windows"] == 0
    if variant != R.RTT_REORDER_UNGUARDED:
        assert plan["tiles_after"] <= plan["tiles_before"]


def test_reorder_variant_checked():
    ctx = R.Context(0)
    with pytest.raises(R.RttError) as e:
        ctx.reorder_plan(_dev(G.laplacian_2d(8)), 6)
    assert e.value.status == 1
    ctx.close()


@pytest.mark.parametrize("case", ["scrambled_band", "scrambled_band_2k", "rmat_10"])
def test_product_through_reordered_operands(case, orc):
    """A' = P A Q^T, B' = Q A, C' = A' B' = P C: C restored from C' by rows."""
    A = CASES[case]()
    ctx = R.Context(0)
    a = _dev(A)
    plan = ctx.reorder_plan(a)
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x, np.int32)).to(DEV)
    a2 = ctx.permute(a, t(plan["row_new_to_old"]), t(plan["inner_old_to_new"]))
    b2 = ctx.permute(a, t(plan["inner_new_to_old"]), None)
    nnz, _ = ctx.symbolic(a2, b2)
    rp = torch.empty(A.m + 1, dtype=torch.int32, device=DEV)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=DEV)
    va = torch.empty(max(nnz, 1), dtype=torch.float64, device=DEV)
    ctx.numeric(rp, ci, va)
    c2 = (A.m, A.n, rp, ci[:nnz], va[:nnz])
    C = _host(ctx.permute(c2, t(plan["row_old_to_new"]), None))
    ctx.close()
    erp, ecol, evals, eabs = orc.spgemm_csr(A, A)
    assert_csr_close(C.rowptr, C.col, C.val, erp, ecol, evals, eabs, f"{case} reordered: ")
    if case.startswith("scrambled"):
        assert plan["accepted"] and plan["tiles_after"] < plan["tiles_before"] // 2


def test_permute_rejects_non_permutations():
    A = G.laplacian_2d(8)
    ctx = R.Context(0)
    bad = torch.zeros(A.m, dtype=torch.int32, device=DEV)  # every row from row 0
    with pytest.raises(R.RttError):
        ctx.permute(_dev(A), bad, None)
    out = torch.arange(A.n, dtype=torch.int32, device=DEV) + 1  # column n out of range
    with pytest.raises(R.RttError):
        ctx.permute(_dev(A), None, out)
    ctx.close()
