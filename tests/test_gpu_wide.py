"""GPU parity of the 64-bit products (rtt_spgemm_symbolic64 / _numeric64):
C through chunks of A's tile rows, int64 row pointer.  Lowered chunk caps
(rtt_config chunk_tiles, chunk_nnz) force many chunks, and chunks that are
halved because their C holds more entries than the cap; every result equals
the oracle (structure bit-exact, values within 1e-12 (|A||B|)_ij) and, bit
for bit, the 32-bit path's."""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G
from conftest import assert_csr_close

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev(A):
    d = torch.device("cuda:0")
    return (A.m, A.n, torch.from_numpy(A.rowptr).to(d), torch.from_numpy(A.col).to(d),
            torch.from_numpy(A.val).to(d))


def _run32(A, B=None, op=R.RTT_OP_AB):
    ctx = R.Context(0)
    da, db = _dev(A), (_dev(B) if B is not None else None)
    nnz, _ = ctx.symbolic(da, db, op)
    d = torch.device("cuda:0")
    rp = torch.empty(A.m + 1, dtype=torch.int32, device=d)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=d)
    va = torch.empty(max(nnz, 1), dtype=torch.float64, device=d)
    ctx.numeric(rp, ci, va)
    torch.cuda.synchronize()
    ctx.close()
    return rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy()


def _run64(A, B=None, op=R.RTT_OP_AB, cfg=None):
    ctx = R.Context(0, cfg)
    da, db = _dev(A), (_dev(B) if B is not None else None)
    nnz = ctx.symbolic64(da, db, op)
    d = torch.device("cuda:0")
    rp = torch.full((A.m + 1,), -7, dtype=torch.int64, device=d)
    ci = torch.full((max(nnz, 1),), -7, dtype=torch.int32, device=d)
    va = torch.full((max(nnz, 1),), float("nan"), dtype=torch.float64, device=d)
    ctx.numeric64(rp, ci, va)
    torch.cuda.synchronize()
    st = ctx.stats()
    ctx.close()
    return rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy(), st


CASES = {
    "stencil27_12": (lambda: G.stencil_27(12, 3), R.RTT_OP_AB),
    "rmat_12_aat": (lambda: G.rmat(12, 16, seed=1), R.RTT_OP_AAT),
    "banded": (lambda: G.banded_scatter(3000, 40, seed=9), R.RTT_OP_AB),
    "lap2d_ragged": (lambda: G.laplacian_2d(37, 11), R.RTT_OP_AB),
    "unsorted": (lambda: G.random_csr(300, 300, 0.02, seed=3, sort=False), R.RTT_OP_AB),
}

CAPS = {
    "default": None,
    "tile_chunks": dict(chunk_tiles=40),               # many chunks of few C tiles
    "halved": dict(chunk_tiles=100000, chunk_nnz=40000),  # chunks halved by their entries
}


@pytest.mark.parametrize("cap", list(CAPS))
@pytest.mark.parametrize("case", list(CASES))
def test_wide_equals_oracle_and_32bit(case, cap, orc):
    make, op = CASES[case]
    A = make()
    rp, ci, va, st = _run64(A, None, op, CAPS[cap])
    B = A.transpose() if op == R.RTT_OP_AAT else A
    assert_csr_close(rp, ci, va, *orc.spgemm_csr(A, B), f"{case}/{cap}: ")
    assert st["nnz_cub"] == orc.nnzcub(A, B)
    prp, pci, pva = _run32(A, None, op)
    assert np.array_equal(rp, prp.astype(np.int64)) and np.array_equal(ci, pci)
    assert np.array_equal(va.view(np.int64), pva.view(np.int64)), f"{case}/{cap}: values"


def test_wide_general_ab(orc):
    A = G.random_csr(500, 300, 0.02, seed=31)
    B = G.random_csr(300, 700, 0.015, seed=32)
    rp, ci, va, _ = _run64(A, B, R.RTT_OP_AB, dict(chunk_tiles=8))
    assert_csr_close(rp, ci, va, *orc.spgemm_csr(A, B), "wide A*B: ")


def test_wide_tile_row_past_the_cap():
    """A single tile row of C holding more entries than chunk_nnz cannot be
    cut further: a clean RTT_ERR_UNREPRESENTABLE."""
    A = G.stencil_27(8, 1)
    ctx = R.Context(0, dict(chunk_nnz=100))
    with pytest.raises(R.RttError) as e:
        ctx.symbolic64(_dev(A))
    assert e.value.status == 6  # RTT_ERR_UNREPRESENTABLE
    ctx.close()


def test_wide_empty():
    A = G.CSR(0, 0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    rp, ci, va, _ = _run64(A)
    assert rp.tolist() == [0] and ci.size == 0
