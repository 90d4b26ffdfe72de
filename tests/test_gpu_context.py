"""GPU: rtt_context_trim releases a context's grown device buffers; the
context stays usable and gives bitwise the same products afterwards."""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _product(ctx, da, m):
    nnz, _ = ctx.symbolic(da)
    d = torch.device("cuda:0")
    rp = torch.empty(m + 1, dtype=torch.int32, device=d)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=d)
    va = torch.empty(max(nnz, 1), dtype=torch.float64, device=d)
    ctx.numeric(rp, ci, va)
    torch.cuda.synchronize()
    return rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy()


def test_trim_releases_and_keeps_results():
    A = G.stencil_27(40, 6)
    d = torch.device("cuda:0")
    da = (A.m, A.n, torch.from_numpy(A.rowptr).to(d), torch.from_numpy(A.col).to(d),
          torch.from_numpy(A.val).to(d))
    ctx = R.Context(0)
    first = _product(ctx, da, A.m)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    ctx.trim()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after > free_before  # the grown buffers went back to the device
    with pytest.raises(R.RttError) as e:  # the symbolic state went with them
        ctx.numeric(*(torch.empty(1, dtype=t, device=d)
                      for t in (torch.int32, torch.int32, torch.float64)))
    assert e.value.status == 11
    again = _product(ctx, da, A.m)
    for x, y in zip(first[:2], again[:2]):
        assert np.array_equal(x, y)
    assert np.array_equal(first[2].view(np.int64), again[2].view(np.int64))
    ctx.close()
