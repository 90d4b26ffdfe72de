"""CPU: pin the oracle restatement (oracle/oracle.c) against the reference's
own CPU code (compiled from its sources into oracle/_ref) and against the
committed golden fixtures generated from it (tests/golden/make_golden.py).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from rtt_spgemm import generators as G
from conftest import assert_tiles_equal

GOLDEN = Path(__file__).resolve().parent / "golden"

CASES = {
    "lap2d_16": lambda: G.laplacian_2d(16),
    "lap2d_ragged": lambda: G.laplacian_2d(13, 7),
    "rand_sorted": lambda: G.random_csr(100, 100, 0.05, seed=1),
    "rand_rect": lambda: G.random_csr(37, 53, 0.1, seed=2),
    "unsorted": lambda: G.random_csr(50, 50, 0.1, seed=3, sort=False),
    "duplicates": lambda: G.random_csr(50, 50, 0.1, seed=4, duplicates=0.3),
    "stencil27_6": lambda: G.stencil_27(6, 1),
    "rmat_8": lambda: G.rmat(8, 8, seed=2),
    "empty_7x9": lambda: G.CSR(7, 9, np.zeros(8, np.int32), np.zeros(0, np.int32), np.zeros(0)),
}
ROW_KEYS = ["tilem", "tilen", "numtile", "tile_ptr", "tile_columnidx", "tile_rowidx", "tile_nnz",
            "tile_csr_Ptr", "tile_csr_Col", "tile_csr_Value", "mask"]
COL_KEYS = ["tilem", "tilen", "numtile", "tile_ptr", "tile_columnidx", "tile_rowidx", "tile_nnz",
            "tile_csr_Ptr", "tile_csr_Col", "tile_csr_Value", "mask", "csc_tile_ptr",
            "csc_tile_rowidx"]
C_KEYS = ["tile_ptr", "tile_columnidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col",
          "tile_csr_Value", "numtile", "nnz"]


@pytest.mark.parametrize("case", list(CASES))
def test_csr2tile_restatement_matches_reference(case, orc, ref):
    A = CASES[case]()
    assert_tiles_equal(orc.csr2tile_row_major(A), ref.csr2tile_row_major(A), ROW_KEYS, case)
    assert_tiles_equal(orc.csr2tile_col_major(A), ref.csr2tile_col_major(A), COL_KEYS, case)


@pytest.mark.parametrize("case", [k for k in CASES if k not in ("rand_rect", "empty_7x9")])
def test_spgemm_restatement_matches_reference(case, orc, ref):
    """With the step-3 quirk reproduced the restatement equals spgemm_cpu bit
    for bit (values included: both sum in the same order without FMA)."""
    A = CASES[case]()
    ra, rb = ref.csr2tile_row_major(A), ref.csr2tile_col_major(A)
    want = ref.spgemm_cpu(ra, rb)
    got = orc.spgemm_tile(orc.csr2tile_row_major(A), orc.csr2tile_col_major(A), quirk=True)
    assert_tiles_equal(got, want, C_KEYS, case)


def test_step3_quirk_only_changes_ragged_tile_counts(orc, ref):
    """On a ragged shape the quirk inflates step-3 counts (tile_nnz) only; the
    entries step 4 writes are the fixed semantics' entries."""
    A = G.random_csr(100, 100, 0.05, seed=1)  # n % 16 == 4
    oa, ob = orc.csr2tile_row_major(A), orc.csr2tile_col_major(A)
    fixed = orc.spgemm_tile(oa, ob, quirk=False)
    quirk = orc.spgemm_tile(oa, ob, quirk=True)
    assert np.array_equal(fixed["tile_ptr"], quirk["tile_ptr"])
    assert np.array_equal(fixed["tile_columnidx"], quirk["tile_columnidx"])
    assert not np.array_equal(fixed["tile_nnz"], quirk["tile_nnz"])
    # every quirk tile holds the fixed tile's entries first, then zero padding
    for s in range(fixed["numtile"]):
        fb, fe = fixed["tile_nnz"][s], fixed["tile_nnz"][s + 1]
        qb = quirk["tile_nnz"][s]
        assert np.array_equal(fixed["tile_csr_Value"][fb:fe], quirk["tile_csr_Value"][qb:qb + fe - fb])


@pytest.mark.parametrize("case", ["lap2d_16", "rmat_8", "duplicates", "lap2d_ragged"])
def test_tile2csr_restatement_matches_reference(case, orc, ref):
    A = CASES[case]()
    c16 = orc.spgemm_tile(orc.csr2tile_row_major(A), orc.csr2tile_col_major(A))
    c8 = orc.tile16_to_tile8(c16)
    for canonical in (True, False):
        got = orc.tile2csr(c8, 8, canonical)
        want = ref.tile2csr(c8, canonical)
        assert np.array_equal(got.rowptr, want.rowptr) and np.array_equal(got.col, want.col)
        assert np.array_equal(got.val, want.val)
    perm = np.random.default_rng(1).permutation(A.m).astype(np.int32)
    got = orc.tile2csr(c8, 8, True, new_to_old=perm)
    want = ref.tile2csr(c8, True, new_to_old=perm)
    assert np.array_equal(got.rowptr, want.rowptr) and np.array_equal(got.col, want.col)


@pytest.mark.parametrize("case", ["lap2d_16", "rmat_8", "duplicates", "stencil27_6"])
def test_row_spa_matches_reference_serialref(case, orc, ref):
    """FP64 row SPA vs the reference's spgemm_serialref (dense-row SPA)."""
    A = CASES[case]()
    rp, col, val, _ = orc.spgemm_csr(A, A, with_abs=False)
    wrp, wcol, wval = ref.spgemm_serialref(A, A)
    assert np.array_equal(rp, wrp.astype(np.int64)) and np.array_equal(col, wcol)
    assert np.array_equal(val, wval)


def test_tile_product_equals_row_spa(orc):
    """The tile path and the row SPA agree on structure (tile2csr of C)."""
    A = G.stencil_27(6, 2)
    c16 = orc.spgemm_tile(orc.csr2tile_row_major(A), orc.csr2tile_col_major(A))
    csr = orc.tile2csr(c16, 16, True)
    rp, col, val, ab = orc.spgemm_csr(A, A)
    assert np.array_equal(csr.rowptr.astype(np.int64), rp) and np.array_equal(csr.col, col)
    assert np.all(np.abs(csr.val - val) <= 1e-12 * ab)


def _golden_files():
    return sorted(GOLDEN.glob("*.npz"))


@pytest.mark.parametrize("path", _golden_files(), ids=lambda p: p.stem)
def test_oracle_matches_golden_fixture(path, orc):
    """Fixtures hold the reference's own outputs; the oracle must reproduce them."""
    z = np.load(path)
    A = G.CSR(int(z["m"]), int(z["n"]), z["rowptr"], z["col"], z["val"])
    rm = orc.csr2tile_row_major(A)
    cm = orc.csr2tile_col_major(A)
    for k in ROW_KEYS[3:]:
        assert np.array_equal(rm[k], z["row_" + k]), k
    for k in COL_KEYS[3:]:
        assert np.array_equal(cm[k], z["col_" + k]), k
    if "c_tile_ptr" in z:
        c = orc.spgemm_tile(rm, cm, quirk=bool(z["quirk"]))
        for k in ("tile_ptr", "tile_columnidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col",
                  "tile_csr_Value"):
            assert np.array_equal(c[k], z["c_" + k]), k


def test_golden_fixtures_present():
    assert len(_golden_files()) >= 4


def test_kat_2d_closed_form_nnz(orc):
    A = G.laplacian_2d(256)
    assert A.nnz == 326656
    rp, _, _, _ = orc.spgemm_csr(A, A, with_abs=False)
    assert rp[-1] == 846852
    assert orc.nnzcub(A, A) == 1629192


# ---------------------------------------------------------------- hybrid leaf tiles
def _kat_a():
    """The worked example of the reference's design document (section 10):
    A's reordered entries (0,0)=a, (1,1)=c, (2,4)=b, (3,5)=d in 8x4 tiles."""
    return G.CSR(4, 8, np.array([0, 1, 2, 3, 4], np.int32), np.array([0, 1, 4, 5], np.int32),
                 np.array([1.0, 3.0, 2.0, 4.0]))


def _assert_hybrid_equal(got, want, tag="", exact=True):
    for k in ("rows", "cols", "tile_rows", "tile_cols", "tile_row_count", "tile_col_count",
              "num_tiles", "payload_size", "dense_tiles", "sparse_tiles"):
        assert got[k] == want[k], f"{tag}{k}: {got[k]} != {want[k]}"
    for k in ("tile_row_ptr", "tile_col_idx", "value_offsets", "masks", "tile_col_ptr",
              "tile_row_idx", "csc_tile_ids"):
        g, w = got[k], want[k]
        if w is None or len(w) == 0:
            assert g is None or len(g) == 0, f"{tag}{k}"
            continue
        assert np.array_equal(g, w), f"{tag}{k} differs"
    gv = got["values"] if got["values"] is not None else np.zeros(0)
    wv = want["values"] if want["values"] is not None else np.zeros(0)
    if exact:
        assert np.array_equal(gv.view(np.int64), wv.view(np.int64)), f"{tag}values"
    else:
        assert np.allclose(gv, wv, rtol=1e-12, atol=1e-12), f"{tag}values"


def test_hybrid_kat_oracle(orc):
    h = orc.csr_to_hybrid_tiles(_kat_a(), 8, 4, False, 24)
    assert list(h["tile_row_ptr"]) == [0, 2] and list(h["tile_col_idx"]) == [0, 1]
    assert list(h["value_offsets"]) == [0, 2, 4]
    assert list(h["masks"]) == [0x00000021, 0x00002100]
    assert list(h["values"]) == [1.0, 3.0, 2.0, 4.0]  # [a, c, b, d]


HYB_CASES = [
    ("a_8x4", 8, 4, False, 24, True),
    ("b_4x8", 4, 8, True, 24, True),
    ("dense_all", 8, 4, False, 1, False),
    ("dense_none", 4, 8, True, 32, True),
    ("thin_2x16", 2, 16, False, 12, True),
]


@pytest.mark.parametrize("cfg", HYB_CASES, ids=[c[0] for c in HYB_CASES])
@pytest.mark.parametrize("mat", ["stencil", "ragged", "dense", "empty_rows"])
def test_hybrid_oracle_matches_reference(ref, orc, cfg, mat):
    A = {"stencil": lambda: G.stencil_27(5, 2), "ragged": lambda: G.laplacian_2d(13, 7),
         "dense": lambda: G.random_csr(37, 29, 0.6, seed=8),
         "empty_rows": lambda: G.random_csr(50, 70, 0.01, seed=9)}[mat]()
    _, tr, tc, cm, thr, csc = cfg
    _assert_hybrid_equal(orc.csr_to_hybrid_tiles(A, tr, tc, cm, thr, csc),
                         ref.csr_to_hybrid_tiles(A, tr, tc, cm, thr, csc), f"{mat}/{cfg[0]}: ")


def test_hybrid_kat_reference(ref):
    h = ref.csr_to_hybrid_tiles(_kat_a(), 8, 4, False, 24)
    assert list(h["masks"]) == [0x00000021, 0x00002100]
    assert list(h["values"]) == [1.0, 3.0, 2.0, 4.0]


def test_hybrid_duplicates_summed(ref, orc):
    A = G.random_csr(40, 40, 0.1, seed=12, duplicates=0.3)
    _assert_hybrid_equal(orc.csr_to_hybrid_tiles(A, 8, 4, False, 4, True),
                         ref.csr_to_hybrid_tiles(A, 8, 4, False, 4, True), "dups: ", exact=False)


# ---------------------------------------------------------------- tail-queue planner
TAIL_POLICY = dict(enabled=1, admission_threshold=256.0, chunk_target=256.0, max_chunks=8,
                   max_heavy_fraction=0.01, record_capacity=1 << 20,
                   workspace_limit_bytes=1 << 30, workspace_reduction=1)
TAIL_MODEL = dict(intercept=0.0, scan=1.0, match=8.0, output=0.25)


def tail_tasks(n, seed, heavy_rate=0.01, invalid_at=None):
    rng = np.random.default_rng(seed)
    scans = rng.integers(0, 40, n)
    heavy = rng.random(n) < heavy_rate
    scans[heavy] = rng.integers(40, 5000, heavy.sum())
    matches = (scans * rng.random(n)).astype(np.int64)
    out = rng.integers(0, 65, n)
    if invalid_at is not None:
        matches[invalid_at] = scans[invalid_at] + 1
    return scans, matches, out


TAIL_CASES = {
    "default": (dict(), dict(), dict(n=5000, seed=1)),
    "enabled": (dict(max_heavy_fraction=0.5), dict(), dict(n=5000, seed=2, heavy_rate=0.02)),
    "fraction_gate": (dict(), dict(), dict(n=3000, seed=3, heavy_rate=0.2)),
    "zero_heavy": (dict(admission_threshold=1e9), dict(), dict(n=1000, seed=4)),
    "workspace_gate": (dict(max_heavy_fraction=1.0, workspace_limit_bytes=4096), dict(), dict(n=2000, seed=5)),
    "record_capacity": (dict(max_heavy_fraction=1.0, record_capacity=3), dict(), dict(n=2000, seed=6, heavy_rate=0.05)),
    "invalid_task": (dict(max_heavy_fraction=1.0), dict(), dict(n=2000, seed=7, invalid_at=900)),
    "odd_model": (dict(chunk_target=33.3, max_chunks=32, max_heavy_fraction=1.0),
                  dict(scan=0.37, match=3.1), dict(n=4000, seed=8, heavy_rate=0.3)),
    "invalid_policy": (dict(max_chunks=1), dict(), dict(n=100, seed=9)),
}


@pytest.mark.parametrize("case", list(TAIL_CASES))
def test_tail_planner_oracle_matches_reference(ref, case):
    import oracle as O
    pol, mod, tk = TAIL_CASES[case]
    pol, mod = {**TAIL_POLICY, **pol}, {**TAIL_MODEL, **mod}
    s, m, o = tail_tasks(**tk)
    ch, plan = O.plan_tail_queue(s, m, o, pol, mod)
    rch, (reason, summ) = ref.plan_tail_queue(s, m, o, pol, mod)
    assert plan["reason"] == reason
    assert np.array_equal(ch, rch)
    assert [plan["heavy_tasks"], plan["chunks"], plan["descriptor_bytes"],
            plan["partial_workspace_bytes"], plan["heavy_flag_bytes"]] == list(summ)


# ---------------------------------------------------------------- early-split planner
EARLY_CASES = {
    # (policy overrides, sm_count, tasks)
    "default_off": (dict(enabled=0), 148, dict(n=2000, seed=11)),
    "reference_defaults": (dict(enabled=1), 148, dict(n=3000, seed=12)),
    "enabled": (dict(enabled=1, admission_threshold=256.0, chunk_target=256.0,
                     max_heavy_fraction=0.5), 148, dict(n=5000, seed=13, heavy_rate=0.02)),
    "small_gpu": (dict(enabled=1, admission_threshold=256.0, chunk_target=256.0,
                       max_heavy_fraction=0.5), 3, dict(n=5000, seed=14, heavy_rate=0.05)),
    "no_reduction": (dict(enabled=1, admission_threshold=256.0, chunk_target=100.0,
                          max_heavy_fraction=1.0, workspace_reduction=0), 148,
                     dict(n=4000, seed=15, heavy_rate=0.1)),
    "invalid_topology": (dict(enabled=1, admission_threshold=256.0, max_heavy_fraction=0.5), 0,
                         dict(n=500, seed=16)),
    "negative_sms": (dict(enabled=1), -4, dict(n=500, seed=17)),
    "base_fraction_gate": (dict(enabled=1, admission_threshold=256.0, chunk_target=256.0), 148,
                           dict(n=3000, seed=18, heavy_rate=0.2)),
    "base_invalid_task": (dict(enabled=1, admission_threshold=256.0, max_heavy_fraction=1.0), 148,
                          dict(n=2000, seed=19, invalid_at=7)),
}


def early_case(case):
    import oracle as O
    pol, sms, tk = EARLY_CASES[case]
    return {**O.EARLY_SPLIT_POLICY, **pol}, dict(TAIL_MODEL), sms, tail_tasks(**tk)


@pytest.mark.parametrize("case", list(EARLY_CASES))
def test_early_split_oracle_matches_reference(ref, case):
    """dmma_plan_tile_early_split (src/dmma_tile_early_split.h:152) compiled
    from the reference against the oracle restatement: gate reasons, worker
    bounds, byte counts and the admitted chunks per task."""
    import oracle as O
    pol, mod, sms, (s, m, o) = early_case(case)
    ch, plan = O.plan_early_split(s, m, o, pol, mod, sms)
    rch, rplan = ref.plan_early_split(s, m, o, pol, mod, sms)
    assert np.array_equal(ch, rch), case
    for k, v in rplan.items():
        assert plan[k] == v, (case, k, plan[k], v)
