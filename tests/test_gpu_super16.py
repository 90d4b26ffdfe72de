"""GPU parity of rtt_super16_index_build (the reference's build_device_index,
src/super16_symbolic.cuh:2123-2323) against the oracle restatement, which
test_super16_cpu.py pins to the reference's own csr2tile and leaf tiles.
Every array bit-exact, for 8x4 A leaves and 4x8 B leaves (with the parent
CSC), over the leaf tiles of rtt_csr_to_hybrid_tiles; malformed leaf tiles
are refused on the host."""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G

pytestmark = pytest.mark.gpu

MATS = {
    "stencil": lambda: G.stencil_27(9, 2),
    "lap2d_ragged": lambda: G.laplacian_2d(37, 11),
    "rmat": lambda: G.rmat(12, 8, seed=3),
    "dense": lambda: G.random_csr(61, 45, 0.7, seed=8),
    "wide": lambda: G.random_csr(20, 5000, 0.01, seed=10),
    "tall": lambda: G.random_csr(5000, 20, 0.05, seed=11),
    "banded": lambda: G.banded_scatter(20000, 40, seed=9),
    "empty_7x9": lambda: G.CSR(7, 9, np.zeros(8, np.int32), np.zeros(0, np.int32), np.zeros(0)),
    "single": lambda: G.CSR(1, 1, np.array([0, 1], np.int32), np.array([0], np.int32),
                            np.array([2.0])),
}
KEYS = ["role", "rows", "cols", "parent_row_count", "parent_col_count", "parent_count",
        "row_ptr", "col_idx", "child_ptr", "child_mask", "child_leaf_ids", "boolean_row_masks",
        "col_ptr", "row_idx", "csc_parent_ids"]


def _equal(got, want, tag):
    for k in KEYS:
        g, w = got[k], want[k]
        if w is None:
            assert g is None, f"{tag}{k}"
            continue
        if isinstance(w, np.ndarray):
            assert np.array_equal(np.asarray(g, np.uint64), np.asarray(w, np.uint64)), f"{tag}{k}"
        else:
            assert int(g) == int(w), f"{tag}{k}: {g} != {w}"


@pytest.mark.parametrize("role", [R.RTT_SUPER16_A8X4, R.RTT_SUPER16_B4X8])
@pytest.mark.parametrize("mat", list(MATS))
def test_super16_index_matches_oracle(orc, mat, role):
    A = MATS[mat]()
    leaf = (R.csr_to_hybrid_tiles(A, 8, 4, False, 24, False) if role == R.RTT_SUPER16_A8X4
            else R.csr_to_hybrid_tiles(A, 4, 8, True, 24, True))
    _equal(R.super16_index(leaf, role), orc.super16_index(leaf, role), f"{mat}/{role}: ")


def test_super16_refuses_malformed_leaves():
    A = G.random_csr(200, 200, 0.05, seed=1)
    leaf = R.csr_to_hybrid_tiles(A, 8, 4, False, 24, False)
    with pytest.raises(R.RttError):  # geometry of the other role
        R.super16_index(leaf, R.RTT_SUPER16_B4X8)
    with pytest.raises(R.RttError):
        R.super16_index(leaf, 3)
    bad = dict(leaf)
    cols = np.array(leaf["tile_col_idx"])
    r = int(np.argmax(np.diff(leaf["tile_row_ptr"]) >= 2))
    b = int(leaf["tile_row_ptr"][r])
    cols[b], cols[b + 1] = cols[b + 1], cols[b]  # decreasing leaf columns in a leaf row
    bad["tile_col_idx"] = cols
    with pytest.raises(R.RttError):
        R.super16_index(bad, R.RTT_SUPER16_A8X4)
    bad = dict(leaf)
    cols = np.array(leaf["tile_col_idx"])
    cols[0] = leaf["tile_col_count"]  # out of range
    bad["tile_col_idx"] = cols
    with pytest.raises(R.RttError):
        R.super16_index(bad, R.RTT_SUPER16_A8X4)
