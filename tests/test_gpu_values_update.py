"""Values-only updates (rtt_spgemm_numeric_values, the reference's dynamic
"values-only" mode): after one symbolic, products with new values of A (and
B) skip csr2tile's counting and the symbolic phase and give what a full
product with those values gives - bitwise, since the summation order is the
same - for A*A, A*A^T and A*B, across the csr2tile paths (sorted, unsorted,
heavy tile rows)."""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G
from conftest import assert_csr_close

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
DEV = torch.device("cuda:0")


def _dev(A):
    return (A.m, A.n, torch.from_numpy(A.rowptr).to(DEV), torch.from_numpy(A.col).to(DEV),
            torch.from_numpy(A.val).to(DEV))


def _full(A, B=None, op=R.RTT_OP_AB):
    ctx = R.Context(0)
    a, b = _dev(A), (_dev(B) if B is not None else None)
    nnz, _ = ctx.symbolic(a, b, op)
    rp = torch.empty(A.m + 1, dtype=torch.int32, device=DEV)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=DEV)
    va = torch.empty(max(nnz, 1), dtype=torch.float64, device=DEV)
    ctx.numeric(rp, ci, va)
    out = rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy()
    ctx.close()
    return out


def _with_values(A, vals):
    return G.CSR(A.m, A.n, A.rowptr, A.col, vals)


CASES = {
    "stencil": lambda: G.stencil_27(10, 1),
    "unsorted": lambda: G.random_csr(300, 300, 0.02, seed=3, sort=False),
    "rmat_13": lambda: G.rmat(13, 16, seed=1),
    "banded": lambda: G.banded_scatter(3000, 40, seed=9),
}


@pytest.mark.parametrize("op", ["A2", "AAT"])
@pytest.mark.parametrize("case", list(CASES))
def test_values_update_equals_full_product(case, op, orc):
    A = CASES[case]()
    rng = np.random.default_rng(11)
    ctx = R.Context(0)
    a = _dev(A)
    o = R.RTT_OP_AAT if op == "AAT" else R.RTT_OP_AB
    nnz, _ = ctx.symbolic(a, None, o)
    rp = torch.empty(A.m + 1, dtype=torch.int32, device=DEV)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=DEV)
    va = torch.empty(max(nnz, 1), dtype=torch.float64, device=DEV)
    ctx.numeric(rp, ci, va)
    for it in range(2):
        vals = rng.uniform(-1, 1, A.nnz)
        ctx.numeric_values(torch.from_numpy(vals).to(DEV), None, rp, ci, va)
        got = rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy()
        A2 = _with_values(A, vals)
        want = _full(A2, None, o)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
        if not case == "unsorted":  # unsorted B rows accumulate with atomics
            assert np.array_equal(got[2].view(np.int64), want[2].view(np.int64)), it
        B = A2 if op == "A2" else A2.transpose()
        erp, ecol, evals, eabs = orc.spgemm_csr(A2, B)
        assert_csr_close(*got, erp, ecol, evals, eabs, f"{case} {op} update {it}: ")
    ctx.close()


def test_values_update_general_ab(orc):
    A = G.random_csr(200, 150, 0.03, seed=21)
    B = G.random_csr(150, 260, 0.03, seed=22)
    ctx = R.Context(0)
    a, b = _dev(A), _dev(B)
    nnz, _ = ctx.symbolic(a, b)
    rp = torch.empty(A.m + 1, dtype=torch.int32, device=DEV)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=DEV)
    va = torch.empty(max(nnz, 1), dtype=torch.float64, device=DEV)
    ctx.numeric(rp, ci, va)
    rng = np.random.default_rng(5)
    av, bv = rng.uniform(-1, 1, A.nnz), rng.uniform(-1, 1, B.nnz)
    ctx.numeric_values(torch.from_numpy(av).to(DEV), torch.from_numpy(bv).to(DEV), rp, ci, va)
    A2, B2 = _with_values(A, av), _with_values(B, bv)
    erp, ecol, evals, eabs = orc.spgemm_csr(A2, B2)
    assert_csr_close(rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy(),
                     erp, ecol, evals, eabs, "A*B update: ")
    st = ctx.stats()
    assert st["nnz_cub"] == orc.nnzcub(A2, B2)
    ctx.close()


def test_values_update_needs_symbolic():
    ctx = R.Context(0)
    v = torch.zeros(4, dtype=torch.float64, device=DEV)
    with pytest.raises(R.RttError):
        ctx.numeric_values(v, None, torch.zeros(2, dtype=torch.int32, device=DEV),
                           torch.zeros(1, dtype=torch.int32, device=DEV), v)
    ctx.close()
