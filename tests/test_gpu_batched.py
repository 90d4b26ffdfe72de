"""GPU parity of the batched form (rtt_spgemm_batched_symbolic / _numeric):
every instance of one block-diagonal pipeline run equals the FP64 row-SPA
oracle (structure bit-exact, values within 1e-12 (|A||B|)_ij) and, bit for
bit, the same instance run alone through the plain device path."""
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


def _plain(A, B=None):
    ctx = R.Context(0)
    da, db = _dev(A), (_dev(B) if B is not None else None)
    nnz, _ = ctx.symbolic(da, db)
    d = torch.device("cuda:0")
    rp = torch.empty(A.m + 1, dtype=torch.int32, device=d)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=d)
    va = torch.empty(max(nnz, 1), dtype=torch.float64, device=d)
    ctx.numeric(rp, ci, va)
    torch.cuda.synchronize()
    ctx.close()
    return rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy()


def _mixed(with_duplicates=False):
    As = [G.banded_scatter(300, 12, seed=1), G.laplacian_2d(37, 11), G.stencil_27(7, 2),
          G.CSR(0, 0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0)),
          G.rmat(9, 8, seed=4), G.random_csr(1, 1, 1.0, seed=2), G.banded_scatter(2100, 40, seed=3)]
    if with_duplicates:
        As.insert(3, G.random_csr(150, 150, 0.04, seed=6, duplicates=0.2))
    return As


def test_batched_with_repeated_columns(orc):
    """One instance repeats columns: the whole batch accumulates with shared
    atomics; every instance stays within the value bound."""
    As = _mixed(with_duplicates=True)
    ctx = R.Context(0)
    outs = R.spgemm_batched(ctx, [_dev(A) for A in As])
    torch.cuda.synchronize()
    for i, (A, (rp, ci, va)) in enumerate(zip(As, outs)):
        erp, ecol, evals, eabs = orc.spgemm_csr(A, A)
        assert_csr_close(rp.cpu().numpy(), ci.cpu().numpy(), va.cpu().numpy(), erp, ecol, evals,
                         eabs, f"instance {i}: ")
    ctx.close()


def test_batched_square_matches_oracle_and_plain(orc):
    As = _mixed()
    ctx = R.Context(0)
    dev = [_dev(A) for A in As]
    outs = R.spgemm_batched(ctx, dev)
    torch.cuda.synchronize()
    for i, (A, (rp, ci, va)) in enumerate(zip(As, outs)):
        rp, ci, va = rp.cpu().numpy(), ci.cpu().numpy(), va.cpu().numpy()
        erp, ecol, evals, eabs = orc.spgemm_csr(A, A)
        assert_csr_close(rp, ci, va, erp, ecol, evals, eabs, f"instance {i}: ")
        if A.m > 0:
            prp, pci, pva = _plain(A)
            assert np.array_equal(rp, prp) and np.array_equal(ci, pci)
            assert np.array_equal(va.view(np.int64), pva.view(np.int64)), f"instance {i}"
    st = ctx.stats()
    assert st["nnz_cub"] == sum(orc.nnzcub(A, A) for A in As)
    ctx.close()


def test_batched_general_ab(orc):
    pairs = [(G.random_csr(40, 70, 0.05, seed=11), G.random_csr(70, 23, 0.08, seed=12)),
             (G.random_csr(17, 5, 0.3, seed=13), G.random_csr(5, 300, 0.02, seed=14)),
             (G.random_csr(64, 64, 0.02, seed=15), G.random_csr(64, 33, 0.1, seed=16))]
    ctx = R.Context(0)
    outs = R.spgemm_batched(ctx, [_dev(a) for a, _ in pairs], [_dev(b) for _, b in pairs])
    torch.cuda.synchronize()
    for i, ((A, B), (rp, ci, va)) in enumerate(zip(pairs, outs)):
        erp, ecol, evals, eabs = orc.spgemm_csr(A, B)
        assert_csr_close(rp.cpu().numpy(), ci.cpu().numpy(), va.cpu().numpy(), erp, ecol, evals,
                         eabs, f"pair {i}: ")
    ctx.close()


def test_batched_config_instances_and_reuse(orc):
    """A slice of the batched configuration's instance distribution, run twice
    on one context (buffers reused), then a plain product on the same context."""
    As = G.batched_instances(12, 2000, 12000, seed=5)
    ctx = R.Context(0)
    dev = [_dev(A) for A in As]
    for _ in range(2):
        outs = R.spgemm_batched(ctx, dev)
        torch.cuda.synchronize()
    for i in (0, 5, 11):
        rp, ci, va = (t.cpu().numpy() for t in outs[i])
        erp, ecol, evals, eabs = orc.spgemm_csr(As[i], As[i])
        assert_csr_close(rp, ci, va, erp, ecol, evals, eabs, f"config instance {i}: ")
    A = G.laplacian_2d(50)
    da = _dev(A)
    nnz, _ = ctx.symbolic(da)
    assert nnz == orc.spgemm_csr(A, A)[0][-1]
    ctx.close()


def test_batched_rejects_bad_shapes():
    ctx = R.Context(0)
    A = G.random_csr(20, 30, 0.1, seed=1)  # not square: A^2 undefined
    with pytest.raises(R.RttError) as ei:
        ctx.batched_symbolic([_dev(A)])
    assert ei.value.status == 3
    ctx.close()


def _split(rp, ci, va, ms, nnz):
    r0 = e0 = 0
    for m, z in zip(ms, nnz):
        yield rp[r0:r0 + m + 1], ci[e0:e0 + z], va[e0:e0 + z]
        r0 += m + 1
        e0 += z


def test_batched_values_update(orc):
    """rtt_spgemm_batched_numeric_values: new values of every instance with the
    batch's structure kept; every instance equals a plain product with those
    values, bit for bit, and the repeated calls replay a CUDA graph."""
    As = _mixed()
    d = torch.device("cuda:0")
    views = [_dev(A) for A in As]
    ctx = R.Context(0)
    nnz, total = ctx.batched_symbolic(views)
    rp = torch.empty(sum(A.m + 1 for A in As), dtype=torch.int32, device=d)
    ci = torch.empty(max(total, 1), dtype=torch.int32, device=d)
    va = torch.empty(max(total, 1), dtype=torch.float64, device=d)
    ctx.batched_numeric(rp, ci, va)
    vt = [torch.zeros(max(A.nnz, 1), dtype=torch.float64, device=d) for A in As]
    rng = np.random.default_rng(2)
    flags = []
    for it in range(3):
        new = [rng.uniform(-1, 1, A.nnz) for A in As]
        for t, v in zip(vt, new):
            if v.size:
                t[:v.size].copy_(torch.from_numpy(v))
        va.fill_(np.nan)
        ctx.batched_numeric_values(vt, None, rp, ci, va)
        flags.append(ctx.stats()["graph_launched"])
        got = _split(rp.cpu().numpy(), ci.cpu().numpy(), va.cpu().numpy(), [A.m for A in As], nnz)
        for i, (A, v, g) in enumerate(zip(As, new, got)):
            if A.m == 0:
                continue
            A2 = G.CSR(A.m, A.n, A.rowptr, A.col, v)
            prp, pci, pva = _plain(A2)
            assert np.array_equal(g[0], prp) and np.array_equal(g[1], pci), f"{it}/{i}"
            assert np.array_equal(g[2].view(np.int64), pva.view(np.int64)), f"{it}/{i}"
    assert flags == [0, 1, 1], flags
    ctx.close()


def test_batched_values_update_general_ab(orc):
    pairs = [(G.random_csr(40, 70, 0.05, seed=11), G.random_csr(70, 23, 0.08, seed=12)),
             (G.random_csr(17, 5, 0.3, seed=13), G.random_csr(5, 300, 0.02, seed=14))]
    d = torch.device("cuda:0")
    da, db = [_dev(a) for a, _ in pairs], [_dev(b) for _, b in pairs]
    ctx = R.Context(0)
    nnz, total = ctx.batched_symbolic(da, db)
    rp = torch.empty(sum(a.m + 1 for a, _ in pairs), dtype=torch.int32, device=d)
    ci = torch.empty(max(total, 1), dtype=torch.int32, device=d)
    va = torch.empty(max(total, 1), dtype=torch.float64, device=d)
    ctx.batched_numeric(rp, ci, va)
    rng = np.random.default_rng(3)
    na = [rng.uniform(-1, 1, a.nnz) for a, _ in pairs]
    nb = [rng.uniform(-1, 1, b.nnz) for _, b in pairs]
    ta = [torch.from_numpy(v).to(d) for v in na]
    tb = [torch.from_numpy(v).to(d) for v in nb]
    ctx.batched_numeric_values(ta, tb, rp, ci, va)
    got = _split(rp.cpu().numpy(), ci.cpu().numpy(), va.cpu().numpy(), [a.m for a, _ in pairs], nnz)
    for i, ((A, B), g) in enumerate(zip(pairs, got)):
        A2 = G.CSR(A.m, A.n, A.rowptr, A.col, na[i])
        B2 = G.CSR(B.m, B.n, B.rowptr, B.col, nb[i])
        erp, ecol, evals, eabs = orc.spgemm_csr(A2, B2)
        assert_csr_close(g[0], g[1], g[2], erp, ecol, evals, eabs, f"pair {i}: ")
    with pytest.raises(R.RttError):  # a batch of squares has no B to update
        ctx2 = R.Context(0)
        ctx2.batched_symbolic([_dev(G.laplacian_2d(8))])
        try:
            ctx2.batched_numeric_values([torch.zeros(1, dtype=torch.float64, device=d)],
                                        [torch.zeros(1, dtype=torch.float64, device=d)],
                                        rp, ci, va)
        finally:
            ctx2.close()
    ctx.close()
