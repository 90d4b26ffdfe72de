"""GPU parity of the reorder (rtt_reorder_plan_build, the reference's
build_dmma_reorder_plan reduced to its traversal and exact commit rule) and of
rtt_csr_permute: the maps equal the CPU restatement's, the tile counts equal
the oracle's, a plan never has more 8x4 A tiles than the identity, and a
product through reordered operands gives the same C once its rows are
restored."""
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
    A = CASES[case]()
    ctx = R.Context(0)
    plan = ctx.reorder_plan(_dev(A))
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
