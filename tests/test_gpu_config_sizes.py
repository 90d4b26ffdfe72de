"""GPU parity at the configured sizes, through the C ABI against the oracle:

* the 3-D 27-point stencil on a 96^3 grid, C = A^2 (the bench workload; the
  same seed as bench.py), plain product and values-only update;
* the R-MAT generator at 2^16 (16 edges per row), C = A*A^T;
* a sample of the batched configuration's 1,024 instances at their own sizes
  (n log-uniform in [2,000, 200,000]), run as one batch.

Structure bit-exact, values within 1e-12 * (|A||B|)_ij.
"""
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


def _outputs(m, nnz):
    d = torch.device("cuda:0")
    return (torch.full((m + 1,), -7, dtype=torch.int32, device=d),
            torch.full((max(nnz, 1),), -7, dtype=torch.int32, device=d),
            torch.full((max(nnz, 1),), float("nan"), dtype=torch.float64, device=d))


def _host(out, nnz):
    rp, ci, va = out
    return rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy()


def test_stencil27_96_a_squared(orc):
    A = G.stencil_27(96, 0)
    ctx = R.Context(0)
    da = _dev(A)
    nnz, tiles = ctx.symbolic(da)
    assert nnz == 106_496_424
    out = _outputs(A.m, nnz)
    ctx.numeric(*out)
    torch.cuda.synchronize()
    want = orc.spgemm_csr(A, A)
    assert_csr_close(*_host(out, nnz), *want, "stencil 96^3: ")
    assert ctx.stats()["nnz_cub"] == 622_835_864
    del want
    # the same structure with other values (values-only update)
    ctx.symbolic(da)
    ctx.numeric(*out)
    new_vals = da[4] * -0.75 + 0.125
    ctx.numeric_values(new_vals, None, *out)
    torch.cuda.synchronize()
    A2 = G.CSR(A.m, A.n, A.rowptr, A.col, new_vals.cpu().numpy())
    assert_csr_close(*_host(out, nnz), *orc.spgemm_csr(A2, A2), "stencil 96^3 values-only: ")
    ctx.close()


def test_rmat16_a_at(orc):
    A = G.rmat(16, 16, seed=1)
    ctx = R.Context(0)
    da = _dev(A)
    nnz, _ = ctx.symbolic(da, None, R.RTT_OP_AAT)
    out = _outputs(A.m, nnz)
    ctx.numeric(*out)
    torch.cuda.synchronize()
    assert_csr_close(*_host(out, nnz), *orc.spgemm_csr(A, A.transpose()), "R-MAT 2^16 AAT: ")
    ctx.close()


def test_batched_config_sample(orc):
    """16 of the 1,024 instances: the four largest, the four smallest and
    eight drawn at random, batched together."""
    ns, _ = G.batched_shapes(1024)
    order = np.argsort(ns)
    rng = np.random.default_rng(7)
    which = sorted(set(order[:4]) | set(order[-4:]) |
                   set(rng.choice(order[4:-4], size=8, replace=False)))
    As = G.batched_instances(1024, which=which)
    assert max(A.m for A in As) == int(ns.max())
    ctx = R.Context(0)
    outs = R.spgemm_batched(ctx, [_dev(A) for A in As])
    torch.cuda.synchronize()
    for i, A, (rp, ci, va) in zip(which, As, outs):
        assert_csr_close(rp.cpu().numpy(), ci.cpu().numpy(), va.cpu().numpy(),
                         *orc.spgemm_csr(A, A), f"batched instance {i} (n={A.m}): ")
    ctx.close()
