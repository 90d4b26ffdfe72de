"""GPU parity of rtt_csr_to_hybrid_tiles (the reference's csr_to_hybrid_tiles,
src/dmma_tiles.h:243) against the oracle restatement, which is itself pinned
to the reference in test_oracle_pin.py.  Structure and values bit-exact
without repeated coordinates; repeated coordinates are summed, within 1e-12."""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G
from test_oracle_pin import HYB_CASES, _assert_hybrid_equal, _kat_a

pytestmark = pytest.mark.gpu

MATS = {
    "stencil": lambda: G.stencil_27(9, 2),
    "lap2d_ragged": lambda: G.laplacian_2d(37, 11),
    "rmat": lambda: G.rmat(10, 8, seed=3),
    "dense": lambda: G.random_csr(61, 45, 0.7, seed=8),
    "unsorted": lambda: G.random_csr(100, 90, 0.05, seed=4, sort=False),
    "wide": lambda: G.random_csr(20, 5000, 0.01, seed=10),
}


@pytest.mark.parametrize("cfg", HYB_CASES, ids=[c[0] for c in HYB_CASES])
@pytest.mark.parametrize("mat", list(MATS))
def test_hybrid_tiles_match_oracle(orc, cfg, mat):
    A = MATS[mat]()
    _, tr, tc, cm, thr, csc = cfg
    got = R.csr_to_hybrid_tiles(A, tr, tc, cm, thr, csc)
    _assert_hybrid_equal(got, orc.csr_to_hybrid_tiles(A, tr, tc, cm, thr, csc), f"{mat}/{cfg[0]}: ")


def test_hybrid_kat():
    h = R.csr_to_hybrid_tiles(_kat_a(), 8, 4, False, 24)
    assert list(h["tile_row_ptr"]) == [0, 2] and list(h["tile_col_idx"]) == [0, 1]
    assert list(h["value_offsets"]) == [0, 2, 4]
    assert list(h["masks"]) == [0x00000021, 0x00002100]
    assert list(h["values"]) == [1.0, 3.0, 2.0, 4.0]


def test_hybrid_duplicates(orc):
    A = G.random_csr(64, 64, 0.1, seed=12, duplicates=0.3)
    _assert_hybrid_equal(R.csr_to_hybrid_tiles(A, 4, 8, True, 6, True),
                         orc.csr_to_hybrid_tiles(A, 4, 8, True, 6, True), "dups: ", exact=False)


def test_hybrid_empty_and_rejections(orc):
    E = G.CSR(0, 7, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    _assert_hybrid_equal(R.csr_to_hybrid_tiles(E, 8, 4, False, 24, True),
                         orc.csr_to_hybrid_tiles(E, 8, 4, False, 24, True), "empty: ")
    A = G.laplacian_2d(8)
    with pytest.raises(R.RttError) as ei:
        R.csr_to_hybrid_tiles(A, 8, 8, False, 24)  # 64 elements
    assert ei.value.status == 1
    with pytest.raises(R.RttError) as ei:
        R.csr_to_hybrid_tiles(A, 8, 4, False, 33)
    assert ei.value.status == 1
    bad = G.CSR(A.m, A.n, A.rowptr, A.col.copy(), A.val)
    bad.col[3] = A.n + 5
    with pytest.raises(R.RttError) as ei:
        R.csr_to_hybrid_tiles(bad, 8, 4, False, 24)
    assert ei.value.status == 2
