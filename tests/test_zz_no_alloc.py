"""rtt_tile2csr_device_noalloc: device tiles -> caller-owned device CSR with no
allocation.  Checked against the allocating entry point rtt_tile2csr on the
same tiles, two calls in a row (the second reuses the per-device scratch, so
a header that was not cleared between calls would show up there).

The file name sorts last so the entry point also runs after every other GPU
test in the session; it passes alone as well.
"""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TILE_KEYS = ("tile_ptr", "tile_columnidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col",
             "tile_csr_Value")


def _c_tiles(A, dim):
    c = R.spgemm_tile(R.csr2tile_row_major(A), R.csr2tile_col_major(A))
    return c if dim == 16 else R.tile16_to_tile8(c)


def _to_device(t):
    d = torch.device("cuda:0")
    out = {k: t[k] for k in ("m", "n", "tilem", "numtile", "nnz")}
    for k in TILE_KEYS:
        a = np.ascontiguousarray(t[k])
        if a.size == 0:
            a = np.zeros(1, dtype=a.dtype)
        out[k] = torch.from_numpy(a).to(d)
    return out


def _noalloc(dt, canonical, stream=0):
    d = torch.device("cuda:0")
    rp = torch.full((dt["m"] + 1,), -3, dtype=torch.int32, device=d)
    nnz = R.tile2csr_device_noalloc(dt, rp, tile_dim=dt["dim"], canonical=canonical,
                                    stream=stream)
    col = torch.full((max(nnz, 1),), -3, dtype=torch.int32, device=d)
    val = torch.full((max(nnz, 1),), float("nan"), dtype=torch.float64, device=d)
    runs = []
    for _ in range(2):
        rp.fill_(-3)
        col.fill_(-3)
        got = R.tile2csr_device_noalloc(dt, rp, col, val, tile_dim=dt["dim"],
                                        canonical=canonical, stream=stream)
        assert got == nnz
        runs.append((rp.cpu().numpy().copy(), col[:nnz].cpu().numpy().copy(),
                     val[:nnz].cpu().numpy().copy()))
    return nnz, runs


CASES = {
    "lap2d_64": lambda: G.laplacian_2d(64),
    "ragged": lambda: G.laplacian_2d(37, 11),
    "rmat_10": lambda: G.rmat(10, 8, seed=2),
    "stencil27_8": lambda: G.stencil_27(8, 1),
    "empty": lambda: G.CSR(20, 20, np.zeros(21, np.int32), np.zeros(0, np.int32), np.zeros(0)),
}


@pytest.mark.parametrize("canonical", [False, True])
@pytest.mark.parametrize("dim", [16, 8])
@pytest.mark.parametrize("case", list(CASES))
def test_matches_tile2csr_twice(case, dim, canonical):
    A = CASES[case]()
    t = _c_tiles(A, dim)
    want = R.tile2csr(t, tile_dim=dim, canonical=canonical)
    dt = _to_device(t)
    dt["dim"] = dim
    nnz, runs = _noalloc(dt, canonical)
    assert nnz == want.col.shape[0]
    for rp, col, val in runs:
        assert np.array_equal(rp, want.rowptr)
        assert np.array_equal(col, want.col)
        assert np.array_equal(val.view(np.int64), want.val.view(np.int64))


def test_side_stream_and_no_device_memory_growth():
    A = G.stencil_27(10, 4)
    t = _c_tiles(A, 16)
    want = R.tile2csr(t, tile_dim=16, canonical=False)
    dt = _to_device(t)
    dt["dim"] = 16
    s = torch.cuda.Stream()
    d = torch.device("cuda:0")
    rp = torch.empty(A.m + 1, dtype=torch.int32, device=d)
    col = torch.empty(want.col.shape[0], dtype=torch.int32, device=d)
    val = torch.empty(want.col.shape[0], dtype=torch.float64, device=d)
    torch.cuda.synchronize()
    # first call on the device does the one-time scratch lookup
    R.tile2csr_device_noalloc(dt, rp, col, val, 16, False, s.cuda_stream)
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        R.tile2csr_device_noalloc(dt, rp, col, val, 16, False, s.cuda_stream)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.array_equal(rp.cpu().numpy(), want.rowptr)
    assert np.array_equal(col.cpu().numpy(), want.col)
    assert np.array_equal(val.cpu().numpy().view(np.int64), want.val.view(np.int64))


def test_rejections():
    A = G.laplacian_2d(32)
    t = _c_tiles(A, 16)
    dt = _to_device(t)
    d = torch.device("cuda:0")
    rp = torch.empty(A.m + 1, dtype=torch.int32, device=d)
    nnz = R.tile2csr_device_noalloc(dt, rp, tile_dim=16)
    small = torch.empty(max(nnz - 1, 1), dtype=torch.int32, device=d)
    smallv = torch.empty(max(nnz - 1, 1), dtype=torch.float64, device=d)
    with pytest.raises(R.RttError, match="capacity"):
        R.tile2csr_device_noalloc(dt, rp, small, smallv, tile_dim=16)
    big = dict(dt, m=(1 << 25) + 1, tilem=((1 << 25) + 16) // 16)
    with pytest.raises(R.RttError, match="33554432"):
        R.tile2csr_device_noalloc(big, rp, tile_dim=16)
    # tile list pointing past numtile: rejected before any kernel walks it
    bad = dict(dt)
    tp = dt["tile_ptr"].clone()
    tp[-1] = dt["numtile"] + 5
    bad["tile_ptr"] = tp
    with pytest.raises(R.RttError, match="malformed") as ei:
        R.tile2csr_device_noalloc(bad, rp, tile_dim=16)
    assert ei.value.status == 1
    # the entry point still works after the rejections
    col = torch.empty(nnz, dtype=torch.int32, device=d)
    val = torch.empty(nnz, dtype=torch.float64, device=d)
    assert R.tile2csr_device_noalloc(dt, rp, col, val, tile_dim=16) == nnz
