"""CPU: the Super16 parent index restatement (oracle.super16_index, after the
reference's build_device_index, src/super16_symbolic.cuh:2123-2323) pinned
against the reference's own CPU code.  Built over the reference's own leaf
tiles (csr_to_hybrid_tiles), the parents of 8x4 A leaves are the 16x16 tiles
of the reference's csr2tile_row_major (row pointer, columns, and Boolean rows
equal to its MSB-first masks bit-reversed); the parents of 4x8 B leaves carry
the tile CSC of its csr2tile_col_major, with the masks of its column-major
tiles.  Child lists are checked against the leaves themselves."""
from __future__ import annotations

import numpy as np
import pytest

from rtt_spgemm import generators as G

CASES = {
    "lap2d_40": lambda: G.laplacian_2d(40),
    "lap2d_ragged": lambda: G.laplacian_2d(13, 7),
    "rand_rect": lambda: G.random_csr(300, 200, 0.03, seed=1),
    "rmat_9": lambda: G.rmat(9, 8, seed=3),
    "banded": lambda: G.banded_scatter(500, 20, seed=2),
    "stencil27_6": lambda: G.stencil_27(6, 1),
    "empty_7x9": lambda: G.CSR(7, 9, np.zeros(8, np.int32), np.zeros(0, np.int32), np.zeros(0)),
}


def bitrev16(x):
    x = np.asarray(x, np.uint32)
    r = np.zeros_like(x)
    for i in range(16):
        r |= ((x >> i) & 1) << (15 - i)
    return r.astype(np.uint16)


def check_children(x, leaf, role):
    """Every leaf once, in its parent, at the slot of its position."""
    RG, CG = (2, 4) if role == 1 else (4, 2)
    trp = np.asarray(leaf["tile_row_ptr"])
    lrow = np.repeat(np.arange(leaf["tile_row_count"]), np.diff(trp))
    tci = np.asarray(leaf["tile_col_idx"])
    ids = np.asarray(x["child_leaf_ids"], np.int64)
    assert np.array_equal(np.sort(ids), np.arange(leaf["num_tiles"]))
    cp = np.asarray(x["child_ptr"], np.int64)
    prow = np.repeat(np.arange(x["parent_row_count"]), np.diff(np.asarray(x["row_ptr"], np.int64)))
    for p in range(x["parent_count"]):
        kids = ids[cp[p]:cp[p + 1]]
        assert np.all(lrow[kids] // RG == prow[p]) and np.all(tci[kids] // CG == x["col_idx"][p])
        slots = (lrow[kids] % RG) * CG + tci[kids] % CG
        assert np.all(np.diff(slots) > 0)  # leaf row by leaf row, in leaf order
        assert int(np.bitwise_or.reduce(1 << slots)) == int(x["child_mask"][p])


@pytest.mark.parametrize("case", list(CASES))
def test_super16_a_parents_are_reference_tiles(case, orc, ref):
    A = CASES[case]()
    leaf = ref.csr_to_hybrid_tiles(A, 8, 4, False, 24, False)
    x = orc.super16_index(leaf, 1)
    t = ref.csr2tile_row_major(A)
    assert np.array_equal(x["row_ptr"], t["tile_ptr"])
    assert np.array_equal(x["col_idx"], t["tile_columnidx"])
    assert np.array_equal(x["boolean_row_masks"], bitrev16(t["mask"]))
    assert x["col_ptr"] is None
    check_children(x, leaf, 1)


@pytest.mark.parametrize("case", list(CASES))
def test_super16_b_parents_are_reference_csc_tiles(case, orc, ref):
    A = CASES[case]()
    leaf = ref.csr_to_hybrid_tiles(A, 4, 8, True, 24, True)
    x = orc.super16_index(leaf, 2)
    t = ref.csr2tile_row_major(A)
    tb = ref.csr2tile_col_major(A)
    assert np.array_equal(x["row_ptr"], t["tile_ptr"])
    assert np.array_equal(x["col_idx"], t["tile_columnidx"])
    assert np.array_equal(x["col_ptr"], tb["csc_tile_ptr"])
    assert np.array_equal(x["row_idx"], tb["csc_tile_rowidx"])
    rows = np.asarray(x["boolean_row_masks"]).reshape(-1, 16)
    assert np.array_equal(rows[np.asarray(x["csc_parent_ids"], np.int64)],
                          bitrev16(tb["mask"]).reshape(-1, 16))
    check_children(x, leaf, 2)
