"""GPU: a Matrix Market file read by rtt_mmio_read (symmetric: rows come out
unsorted, as from the reference's reader) goes through the device product;
C = A^2 against the oracle, with the file's values and with the reference
benchmark's value overwrite."""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G
from conftest import assert_csr_close

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _write_symmetric(path, A):
    rows = np.repeat(np.arange(A.m), np.diff(A.rowptr))
    keep = A.col <= rows  # lower triangle, the file stores one half
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n")
        f.write(f"{A.m} {A.n} {int(keep.sum())}\n")
        for i, j, v in zip(rows[keep], A.col[keep], A.val[keep]):
            f.write(f"{i + 1} {j + 1} {float(v)!r}\n")


@pytest.mark.parametrize("value_mode", [0, 1])
def test_mmio_file_through_the_device_path(tmp_path, orc, value_mode):
    S = G.stencil_27(10, 5)
    sym = G.from_coo(S.m, S.n, np.repeat(np.arange(S.m), np.diff(S.rowptr)), S.col, S.val)
    rows = np.repeat(np.arange(sym.m), np.diff(sym.rowptr))
    low = sym.col <= rows
    A0 = G.from_coo(sym.m, sym.n, np.concatenate([rows[low], sym.col[low]]),
                    np.concatenate([sym.col[low], rows[low]]),
                    np.concatenate([sym.val[low], sym.val[low]]))  # symmetric values
    path = tmp_path / "s.mtx"
    _write_symmetric(path, A0)
    A = R.mmio_read(path, value_mode)
    assert A.is_symmetric and A.nnz == A0.nnz
    d = torch.device("cuda:0")
    da = (A.m, A.n, torch.from_numpy(A.rowptr).to(d), torch.from_numpy(A.col).to(d),
          torch.from_numpy(A.val).to(d))
    ctx = R.Context(0)
    nnz, _ = ctx.symbolic(da)
    rp = torch.empty(A.m + 1, dtype=torch.int32, device=d)
    ci = torch.empty(max(nnz, 1), dtype=torch.int32, device=d)
    va = torch.empty(max(nnz, 1), dtype=torch.float64, device=d)
    ctx.numeric(rp, ci, va)
    torch.cuda.synchronize()
    assert_csr_close(rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy(),
                     *orc.spgemm_csr(A, A), f"mtx value_mode {value_mode}: ")
    ctx.close()
