"""GPU parity of the dynamic-B modes (rtt_spgemm_update_b; the reference's
B update modes, src/main.cu:26-32 and rebuild_b, :1406-1453): the same A with
a new B (structure mode) or with B's rows permuted (permutation mode), against
the oracle and against fresh products."""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G
from conftest import assert_csr_close

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
DEV = "cuda:0"


def _dev(A):
    d = torch.device(DEV)
    return (A.m, A.n, torch.from_numpy(A.rowptr).to(d), torch.from_numpy(A.col).to(d),
            torch.from_numpy(A.val).to(d))


def _numeric(ctx, m, nnz):
    d = torch.device(DEV)
    rp = torch.full((m + 1,), -7, dtype=torch.int32, device=d)
    ci = torch.full((max(nnz, 1),), -7, dtype=torch.int32, device=d)
    va = torch.full((max(nnz, 1),), float("nan"), dtype=torch.float64, device=d)
    ctx.numeric(rp, ci, va)
    torch.cuda.synchronize()
    return rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy()


def _fresh(A, B):
    ctx = R.Context(0)
    da, db = _dev(A), _dev(B)
    nnz, _ = ctx.symbolic(da, db)
    out = _numeric(ctx, A.m, nnz)
    ctx.close()
    return out


def _permute_rows(B, new_to_old):
    rows = [np.arange(B.rowptr[o], B.rowptr[o + 1]) for o in new_to_old]
    idx = np.concatenate(rows) if rows else np.zeros(0, np.int64)
    rp = np.zeros(B.m + 1, np.int64)
    np.cumsum(np.diff(B.rowptr)[new_to_old], out=rp[1:])
    return G.CSR(B.m, B.n, rp.astype(np.int32), B.col[idx].copy(), B.val[idx].copy())


def _permute_cols(A, old_to_new):
    rows = np.repeat(np.arange(A.m), np.diff(A.rowptr))
    return G.from_coo(A.m, A.n, rows, old_to_new[A.col], A.val)


def test_structure_mode(orc):
    A = G.random_csr(500, 300, 0.02, seed=51)
    B1 = G.random_csr(300, 700, 0.015, seed=52)
    B2 = G.banded_scatter(300, 12, seed=53)
    ctx = R.Context(0)
    da, d1, d2 = _dev(A), _dev(B1), _dev(B2)
    nnz, _ = ctx.symbolic(da, d1)
    got1 = _numeric(ctx, A.m, nnz)
    assert_csr_close(*got1, *orc.spgemm_csr(A, B1), "A*B1: ")
    for B, dB in ((B2, d2), (B1, d1)):  # a new structure, then the first one again
        nnz, _ = ctx.update_b(dB)
        got = _numeric(ctx, A.m, nnz)
        assert_csr_close(*got, *orc.spgemm_csr(A, B), "updated B: ")
        want = _fresh(A, B)
        assert all(np.array_equal(g, w) for g, w in zip(got[:2], want[:2]))
        assert np.array_equal(got[2].view(np.int64), want[2].view(np.int64))
    ctx.close()


def test_permutation_mode(orc):
    """A' = A with columns renumbered by a permutation q; B's rows taken in
    the matching order give B' = Q B, and A' * B' = A * B."""
    A = G.stencil_27(9, 4)
    B = G.banded_scatter(A.n, 10, seed=61)
    rng = np.random.default_rng(62)
    new_to_old = rng.permutation(A.n).astype(np.int32)
    old_to_new = np.empty_like(new_to_old)
    old_to_new[new_to_old] = np.arange(A.n, dtype=np.int32)
    Ap = _permute_cols(A, old_to_new)
    ctx = R.Context(0)
    da, dB = _dev(Ap), _dev(B)
    nnz, _ = ctx.symbolic(da, dB)  # any B first: the permuted one replaces it
    perm = torch.from_numpy(new_to_old).to(DEV)
    nnz, _ = ctx.update_b(dB, perm)
    got = _numeric(ctx, A.m, nnz)
    assert_csr_close(*got, *orc.spgemm_csr(A, B), "permuted B: ")
    want = _fresh(Ap, _permute_rows(B, new_to_old))
    assert all(np.array_equal(g, w) for g, w in zip(got[:2], want[:2]))
    assert np.array_equal(got[2].view(np.int64), want[2].view(np.int64))
    ctx.close()


def test_update_b_errors():
    A = G.random_csr(50, 40, 0.1, seed=71)
    ctx = R.Context(0)
    with pytest.raises(R.RttError) as e:
        ctx.update_b(_dev(G.random_csr(40, 30, 0.1, seed=72)))
    assert e.value.status == 11  # RTT_ERR_STATE: no symbolic phase yet
    da = _dev(A)
    ctx.symbolic(da, _dev(G.random_csr(40, 30, 0.1, seed=73)))
    with pytest.raises(R.RttError) as e:
        ctx.update_b(_dev(G.random_csr(41, 30, 0.1, seed=74)))
    assert e.value.status == 3  # RTT_ERR_SHAPE_MISMATCH
    dB = _dev(G.random_csr(40, 30, 0.1, seed=75))
    bad = torch.zeros(40, dtype=torch.int32, device=DEV)  # not a permutation
    with pytest.raises(R.RttError) as e:
        ctx.update_b(dB, bad)
    assert e.value.status == 8  # RTT_ERR_DEVICE_CHECK
    ctx.close()
    sq = G.random_csr(40, 40, 0.1, seed=76)
    ctx = R.Context(0)
    ctx.symbolic(_dev(sq), None, R.RTT_OP_AAT)
    with pytest.raises(R.RttError) as e:
        ctx.update_b(_dev(sq))
    assert e.value.status == 11  # not after A*A^T
    ctx.close()
