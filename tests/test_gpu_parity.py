"""GPU parity: every drop-in entry point against the CPU oracle (and the
reference's own CPU code where it is built).

Structure (tile pointers, tile columns, per-tile offsets, row offsets, column
bytes, masks, CSR row pointers and columns) must be bit-exact; FP64 values
within 1e-12 * (|A||B|)_ij.
"""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G
from conftest import VALUE_RTOL, assert_csr_close, assert_tiles_equal

pytestmark = pytest.mark.gpu


def _empty(m, n):
    return G.CSR(m, n, np.zeros(m + 1, np.int32), np.zeros(0, np.int32), np.zeros(0))


def _hub_rows(m, n, hubs, hub_len, other_len, seed, dup_every=0):
    """Rows of other_len random sorted columns plus hub rows of hub_len: tile
    rows above 2048 entries take csr2tile's CTA-per-tile-row path.  dup_every
    repeats every dup_every-th hub column a few times (sorted, so the tile
    columns stay non-decreasing)."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(m):
        k = hub_len if i in hubs else other_len
        c = np.sort(rng.choice(n, size=min(k, n), replace=False))
        if dup_every and i in hubs:
            c = np.sort(np.concatenate([c, np.repeat(c[::dup_every], 3)]))
        rows.append(c)
    rp = np.zeros(m + 1, np.int32)
    rp[1:] = np.cumsum([len(c) for c in rows])
    col = np.concatenate(rows).astype(np.int32)
    return G.CSR(m, n, rp, col, rng.uniform(-1, 1, col.size))


CASES = {
    "lap2d_16": lambda: G.laplacian_2d(16),
    "lap2d_64": lambda: G.laplacian_2d(64),
    "lap2d_ragged": lambda: G.laplacian_2d(13, 7),
    "rand_sorted": lambda: G.random_csr(200, 200, 0.03, seed=1),
    "rand_rect": lambda: G.random_csr(37, 53, 0.1, seed=2),
    "unsorted": lambda: G.random_csr(90, 90, 0.08, seed=3, sort=False),
    "duplicates": lambda: G.random_csr(70, 70, 0.08, seed=4, duplicates=0.3),
    "explicit_zeros": lambda: G.random_csr(80, 80, 0.1, seed=5, explicit_zeros=0.3),
    "dense": lambda: G.random_csr(48, 48, 0.9, seed=6),
    "stencil27_8": lambda: G.stencil_27(8, 1),
    "rmat_10": lambda: G.rmat(10, 8, seed=3),
    "banded": lambda: G.banded_scatter(500, 12, seed=5),
    "empty_0x0": lambda: _empty(0, 0),
    "empty_10x10": lambda: _empty(10, 10),
    "one": lambda: G.CSR(1, 1, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([2.5])),
    # heavy tile rows: one pass, many passes (> 2048 tiles), repeated columns,
    # and a column span past the bitmap (back to the half-warp path)
    "hub_rows": lambda: _hub_rows(70, 60000, {3, 17, 40}, 5000, 20, seed=7),
    "hub_many_tiles": lambda: _hub_rows(40, 1000000, {5}, 40000, 30, seed=8),
    "hub_dups": lambda: _hub_rows(40, 20000, {1, 2}, 3000, 10, seed=9, dup_every=5),
    "hub_wide_span": lambda: _hub_rows(20, 3000000, {4}, 6000, 5, seed=10),
}
SQUARE = [k for k in CASES if k != "rand_rect" and not k.startswith("hub")]

ROW_KEYS = ["m", "n", "tilem", "tilen", "numtile", "tile_ptr", "tile_columnidx", "tile_rowidx",
            "tile_nnz", "tile_csr_Ptr", "tile_csr_Col", "tile_csr_Value", "mask"]
COL_KEYS = ROW_KEYS + ["csc_tile_ptr", "csc_tile_rowidx"]
C_KEYS = ["tile_ptr", "tile_columnidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col", "numtile",
          "nnz", "mask", "tile_rowidx"]


@pytest.mark.parametrize("case", list(CASES))
def test_csr2tile_row_major(case, orc):
    A = CASES[case]()
    got = R.csr2tile_row_major(A)
    assert_tiles_equal(got, orc.csr2tile_row_major(A), ROW_KEYS, f"{case}: ")


@pytest.mark.parametrize("case", list(CASES))
def test_csr2tile_col_major(case, orc):
    A = CASES[case]()
    got = R.csr2tile_col_major(A)
    assert_tiles_equal(got, orc.csr2tile_col_major(A), COL_KEYS, f"{case}: ")


def _abs_tiles(t: dict) -> dict:
    u = dict(t)
    u["tile_csr_Value"] = np.abs(t["tile_csr_Value"])
    return u


def _check_spgemm_tile(A, B, orc, tag):
    a, b = R.csr2tile_row_major(A), R.csr2tile_col_major(B)
    got = R.spgemm_tile(a, b)
    oa, ob = orc.csr2tile_row_major(A), orc.csr2tile_col_major(B)
    want = orc.spgemm_tile(oa, ob)
    bound = orc.spgemm_tile(_abs_tiles(oa), _abs_tiles(ob))["tile_csr_Value"]
    assert_tiles_equal(got, want, C_KEYS, tag)
    err = np.abs(got["tile_csr_Value"] - want["tile_csr_Value"])
    assert np.all(err <= VALUE_RTOL * bound), f"{tag}max value error {err.max() if err.size else 0}"
    assert got["m"] == A.m and got["n"] == B.n
    return got


@pytest.mark.parametrize("case", SQUARE)
def test_spgemm_tile_a_squared(case, orc):
    A = CASES[case]()
    _check_spgemm_tile(A, A, orc, f"{case} A*A: ")


@pytest.mark.parametrize("case", ["rand_rect", "rmat_10", "lap2d_ragged", "banded", "duplicates"])
def test_spgemm_tile_a_at(case, orc):
    A = CASES[case]()
    _check_spgemm_tile(A, A.transpose(), orc, f"{case} A*A^T: ")


def test_spgemm_tile_general_ab(orc):
    A = G.random_csr(61, 45, 0.12, seed=11)
    B = G.random_csr(45, 77, 0.09, seed=12, sort=False, duplicates=0.2)
    _check_spgemm_tile(A, B, orc, "A*B: ")


def test_spgemm_tile_matches_reference_cpu(ref, orc):
    """Pin against the reference's spgemm_cpu itself (with the in-tile column
    fix applied at the call site) on a shape where its step-3 row-length quirk
    cannot fire (n % 16 == 0)."""
    A = G.laplacian_2d(32)
    ra, rb = ref.csr2tile_row_major(A), ref.csr2tile_col_major(A)
    want = ref.spgemm_cpu(ra, rb)
    got = R.spgemm_tile(R.csr2tile_row_major(A), R.csr2tile_col_major(A))
    assert_tiles_equal(got, want, ["tile_ptr", "tile_columnidx", "tile_nnz", "tile_csr_Ptr",
                                   "tile_csr_Col", "numtile", "nnz"], "ref spgemm_cpu: ")
    # Laplacian products of small integers are exact in FP64
    assert np.array_equal(got["tile_csr_Value"], want["tile_csr_Value"])


@pytest.mark.parametrize("case", ["lap2d_64", "rmat_10", "duplicates", "lap2d_ragged"])
def test_tile16_to_tile8(case, orc):
    A = CASES[case]()
    c16 = orc.spgemm_tile(orc.csr2tile_row_major(A), orc.csr2tile_col_major(A))
    got = R.tile16_to_tile8(c16)
    want = orc.tile16_to_tile8(c16)
    assert_tiles_equal(got, want, ["m", "n", "tilem", "tilen", "numtile", "nnz", "tile_ptr",
                                   "tile_columnidx", "tile_rowidx", "tile_nnz", "tile_csr_Ptr",
                                   "tile_csr_Col", "tile_csr_Value"], f"{case}: ")


@pytest.mark.parametrize("case", ["lap2d_64", "rmat_10", "duplicates", "lap2d_ragged", "one"])
@pytest.mark.parametrize("canonical", [True, False])
def test_tile2csr_8x8_matches_reference(case, canonical, orc, ref):
    A = CASES[case]()
    c16 = orc.spgemm_tile(orc.csr2tile_row_major(A), orc.csr2tile_col_major(A))
    c8 = orc.tile16_to_tile8(c16)
    got = R.tile2csr(c8, tile_dim=8, canonical=canonical)
    want = ref.tile2csr(c8, canonical=canonical)
    assert np.array_equal(got.rowptr, want.rowptr)
    assert np.array_equal(got.col, want.col)
    assert np.array_equal(got.val, want.val)


@pytest.mark.parametrize("case", ["lap2d_64", "unsorted", "lap2d_ragged", "empty_10x10"])
def test_tile2csr_16(case, orc):
    A = CASES[case]()
    c16 = orc.spgemm_tile(orc.csr2tile_row_major(A), orc.csr2tile_col_major(A))
    got = R.tile2csr(c16, tile_dim=16, canonical=True)
    want = orc.tile2csr(c16, 16, canonical=True)
    assert np.array_equal(got.rowptr, want.rowptr)
    assert np.array_equal(got.col, want.col)
    assert np.array_equal(got.val, want.val)


def test_tile2csr_noncanonical_sorts_like_reference(orc, ref):
    """Shuffle entries inside tile rows (with duplicate columns) so the heap
    sort of the non-canonical path does real work; must match the reference."""
    A = G.random_csr(64, 64, 0.2, seed=21, duplicates=0.25)
    c16 = orc.spgemm_tile(orc.csr2tile_row_major(A), orc.csr2tile_col_major(A))
    c8 = orc.tile16_to_tile8(c16)
    rng = np.random.default_rng(3)
    for t in range(c8["numtile"]):
        b, e = c8["tile_nnz"][t], c8["tile_nnz"][t + 1]
        for r in range(8):
            s = b + c8["tile_csr_Ptr"][t * 8 + r]
            f = e if r == 7 else b + c8["tile_csr_Ptr"][t * 8 + r + 1]
            p = rng.permutation(f - s) + s
            c8["tile_csr_Col"][s:f] = c8["tile_csr_Col"][p]
            c8["tile_csr_Value"][s:f] = c8["tile_csr_Value"][p]
    got = R.tile2csr(c8, tile_dim=8, canonical=False)
    want = ref.tile2csr(c8, canonical=False)
    assert np.array_equal(got.rowptr, want.rowptr)
    assert np.array_equal(got.col, want.col)
    assert np.array_equal(got.val, want.val)


def test_tile2csr_restore_rows(orc, ref):
    A = G.laplacian_2d(24)
    c16 = orc.spgemm_tile(orc.csr2tile_row_major(A), orc.csr2tile_col_major(A))
    c8 = orc.tile16_to_tile8(c16)
    perm = np.random.default_rng(7).permutation(A.m).astype(np.int32)
    got = R.tile2csr(c8, tile_dim=8, canonical=True, new_to_old=perm)
    want = ref.tile2csr(c8, canonical=True, new_to_old=perm)
    assert np.array_equal(got.rowptr, want.rowptr)
    assert np.array_equal(got.col, want.col)
    assert np.array_equal(got.val, want.val)
    # illegal permutation (duplicate target) is rejected
    bad = perm.copy()
    bad[1] = bad[0]
    with pytest.raises(R.RttError) as e:
        R.tile2csr(c8, tile_dim=8, new_to_old=bad)
    assert e.value.status == 9
    # a shortened prefix with non-empty rows after it is rejected
    with pytest.raises(R.RttError) as e:
        R.tile2csr(c8, tile_dim=8, new_to_old=perm[: A.m // 2], perm_size=A.m // 2)
    assert e.value.status == 10


def test_invalid_csr_rejected():
    A = G.laplacian_2d(8)
    A.col[5] = A.n + 3
    with pytest.raises(R.RttError) as e:
        R.csr2tile_row_major(A)
    assert e.value.status == 2


def _with_long_row(n=2000, width=900, seed=5):
    """Random CSR whose row 37 holds `width` sorted columns (the validation's
    warp-wide walk of rows longer than 256 entries)."""
    A = G.random_csr(n, n, 0.002, seed=seed)
    rows = [A.col[A.rowptr[i]:A.rowptr[i + 1]] for i in range(n)]
    vals = [A.val[A.rowptr[i]:A.rowptr[i + 1]] for i in range(n)]
    rng = np.random.default_rng(seed)
    rows[37] = np.sort(rng.choice(n, width, replace=False)).astype(np.int32)
    vals[37] = rng.uniform(-1, 1, width)
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    return G.CSR(n, n, rp, np.concatenate(rows).astype(np.int32), np.concatenate(vals))


def test_long_row_validation(orc):
    """A row of 900 entries: sorted, with two columns swapped (generic
    path), with a repeated column, and with a column out of range."""
    A = _with_long_row()
    assert_tiles_equal(R.csr2tile_row_major(A), orc.csr2tile_row_major(A), ROW_KEYS, "long row: ")
    b = int(A.rowptr[37])
    U = G.CSR(A.m, A.n, A.rowptr, A.col.copy(), A.val)
    U.col[b + 100], U.col[b + 500] = U.col[b + 500], U.col[b + 100]  # tile columns decrease
    assert_tiles_equal(R.csr2tile_row_major(U), orc.csr2tile_row_major(U), ROW_KEYS, "unsorted: ")
    D = G.CSR(A.m, A.n, A.rowptr, A.col.copy(), A.val)
    D.col[b + 301] = D.col[b + 300]  # repeated column (still non-decreasing)
    assert_tiles_equal(R.csr2tile_row_major(D), orc.csr2tile_row_major(D), ROW_KEYS, "repeat: ")
    X = G.CSR(A.m, A.n, A.rowptr, A.col.copy(), A.val)
    X.col[b + 700] = A.n + 1
    with pytest.raises(R.RttError) as e:
        R.csr2tile_row_major(X)
    assert e.value.status == 2


def test_malformed_tiles_rejected(orc):
    A = G.laplacian_2d(16)
    a = orc.csr2tile_row_major(A)
    b = orc.csr2tile_col_major(A)
    b["tile_nnz"] = b["tile_nnz"].copy()
    b["tile_nnz"][3] = b["tile_nnz"][4] + 5  # not monotone
    with pytest.raises(R.RttError) as e:
        R.spgemm_tile(a, b)
    assert e.value.status == 1
