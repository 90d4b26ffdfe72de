"""GPU parity of the device-resident CSR -> CSR product (the timed path):
csr2tile(A, B) -> symbolic -> numeric (fused tile2csr or separate) against the
FP64 row-SPA oracle.  Structure bit-exact, values within 1e-12 * (|A||B|)_ij.
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


def _run(ctx, A, B=None, op=R.RTT_OP_AB):
    # the operands stay borrowed until numeric() returns: keep them alive here
    da = _dev(A)
    db = _dev(B) if B is not None else None
    nnz, tiles = ctx.symbolic(da, db, op)
    d = torch.device("cuda:0")
    rp = torch.full((A.m + 1,), -7, dtype=torch.int32, device=d)
    ci = torch.full((max(nnz, 1),), -7, dtype=torch.int32, device=d)
    va = torch.full((max(nnz, 1),), float("nan"), dtype=torch.float64, device=d)
    ctx.numeric(rp, ci, va)
    torch.cuda.synchronize()
    return rp.cpu().numpy(), ci[:nnz].cpu().numpy(), va[:nnz].cpu().numpy(), nnz, tiles


CASES = {
    "lap2d_256": lambda: G.laplacian_2d(256),
    "lap2d_ragged": lambda: G.laplacian_2d(37, 11),
    "stencil27_12": lambda: G.stencil_27(12, 3),
    "rmat_12": lambda: G.rmat(12, 16, seed=1),
    "banded": lambda: G.banded_scatter(3000, 40, seed=9),
    "banded_wide": lambda: G.banded_scatter(2000, 64, seed=5),  # tile rows > 2048 entries
    "unsorted": lambda: G.random_csr(300, 300, 0.02, seed=3, sort=False),
    "duplicates": lambda: G.random_csr(200, 200, 0.03, seed=4, duplicates=0.3),
    "dense": lambda: G.random_csr(96, 96, 0.85, seed=6),
}

CONFIGS = {
    "fused_dmma": dict(fused_csr_output=1, dmma_pair_cutoff=3072),
    "fused_nodmma": dict(fused_csr_output=1, dmma_pair_cutoff=0),
    "unfused": dict(fused_csr_output=0, dmma_pair_cutoff=3072),
    "all_dmma": dict(fused_csr_output=1, dmma_pair_cutoff=1),
    "flat": dict(fused_csr_output=1, dmma_pair_cutoff=0, b_staging=0),
    "flat_unfused": dict(fused_csr_output=0, dmma_pair_cutoff=0, b_staging=0),
    "staged": dict(fused_csr_output=1, dmma_pair_cutoff=0, b_staging=1),
    # FP64 DMMA straight from 8x4 / 4x8 hybrid leaves
    "leaf": dict(leaf_dmma=1),
}


@pytest.mark.parametrize("cfg", list(CONFIGS))
@pytest.mark.parametrize("case", list(CASES))
def test_a_squared(case, cfg, orc):
    A = CASES[case]()
    ctx = R.Context(0, CONFIGS[cfg])
    rp, ci, va, nnz, tiles = _run(ctx, A)
    erp, ecol, evals, eabs = orc.spgemm_csr(A, A)
    assert_csr_close(rp, ci, va, erp, ecol, evals, eabs, f"{case}/{cfg}: ")
    st = ctx.stats()
    assert st["nnz_c"] == nnz
    assert st["nnz_cub"] == orc.nnzcub(A, A)
    if cfg == "all_dmma" and nnz > 0:
        # every pair qualifies; B tile rows wider than the per-step table
        # (64 tiles) still take the sparse path
        assert st["dmma_pairs"] > 0
    if cfg in ("fused_nodmma", "flat", "flat_unfused", "staged"):
        assert st["dmma_pairs"] == 0
    if cfg == "leaf" and nnz > 0:
        assert st["dmma_pairs"] > 0  # leaf pairs multiplied on the tensor cores
    ctx.close()


@pytest.mark.parametrize("case", ["rmat_12", "lap2d_ragged", "banded", "unsorted"])
def test_a_at(case, orc):
    A = CASES[case]()
    ctx = R.Context(0)
    rp, ci, va, nnz, _ = _run(ctx, A, None, R.RTT_OP_AAT)
    At = A.transpose()
    erp, ecol, evals, eabs = orc.spgemm_csr(A, At)
    assert_csr_close(rp, ci, va, erp, ecol, evals, eabs, f"{case} AAT: ")
    ctx.close()


def test_general_ab(orc):
    A = G.random_csr(500, 300, 0.02, seed=31)
    B = G.random_csr(300, 700, 0.015, seed=32)
    ctx = R.Context(0)
    rp, ci, va, nnz, _ = _run(ctx, A, B)
    erp, ecol, evals, eabs = orc.spgemm_csr(A, B)
    assert_csr_close(rp, ci, va, erp, ecol, evals, eabs, "A*B: ")
    ctx.close()


def test_wide_and_crowded_tile_rows(orc):
    """C tile rows whose tile columns span more than the 8192-column bitmap of
    the symbolic step, and rows with more C tiles than one slot window: both
    are processed in column windows."""
    A = G.random_csr(40, 500, 0.05, seed=41)
    B = G.random_csr(500, 300000, 0.0004, seed=42)
    ctx = R.Context(0)
    rp, ci, va, nnz, tiles = _run(ctx, A, B)
    erp, ecol, evals, eabs = orc.spgemm_csr(A, B)
    assert_csr_close(rp, ci, va, erp, ecol, evals, eabs, "wide A*B: ")
    assert tiles > 2 * 254  # several slot windows per C tile row
    ctx.close()


# C tile rows with more tiles than one slot window (banded plus scatter,
# R-MAT hubs, unsorted random rows): several windows per tile row
MANY_WINDOW_CASES = {
    "banded": CASES["banded"],
    "rmat_12": CASES["rmat_12"],
    "banded_20k": lambda: G.banded_scatter(20000, 24, seed=11),
    "unsorted_wide": lambda: G.random_csr(3000, 3000, 0.01, seed=12, sort=False),
    # hub rows with > 1024 A entries per row pair: symbolic step 2's wide CTA
    "rmat_14": lambda: G.rmat(14, 16, seed=2),
}


@pytest.mark.parametrize("case", list(MANY_WINDOW_CASES))
def test_many_window_rows_fused_equals_tiles(case, orc):
    """C written as CSR directly by the numeric kernel or as tiles converted by
    tile2csr, with heavy tile rows split into window tasks or not: every entry
    is summed in the same order, so all four are bitwise equal, and they match
    the oracle."""
    A = MANY_WINDOW_CASES[case]()
    runs = {}
    for name, cfg in (("fused", dict(fused_csr_output=1)), ("tiled", dict(fused_csr_output=0)),
                      ("fused_split1", dict(fused_csr_output=1, split_target=1)),
                      ("tiled_split1", dict(fused_csr_output=0, split_target=1)),
                      ("fused_split64k", dict(fused_csr_output=1, split_target=1 << 16)),
                      ("fused_nosplit", dict(fused_csr_output=1, split_target=-1)),
                      # heavy rows accumulated in C's values in device memory
                      ("fused_global", dict(fused_csr_output=1, global_rows=1))):
        ctx = R.Context(0, cfg)
        runs[name] = _run(ctx, A)
        # split_target 1: every multi-window row becomes one task per window
        if "split1" in name:
            assert ctx.stats()["split_windows"] > 0, name
        if "nosplit" in name:
            assert ctx.stats()["split_windows"] == 0, name
        # a 2^16 target groups banded_20k's windows: tasks of several windows,
        # whose workers carry per-entry cursors from one window to the next
        if name == "fused_split64k" and case == "banded_20k":
            assert ctx.stats()["split_multi_window_tasks"] > 0, name
        ctx.close()
    fused = runs["fused"]
    for name, other in runs.items():
        assert np.array_equal(fused[0], other[0]) and np.array_equal(fused[1], other[1]), name
        assert np.array_equal(fused[2].view(np.int64), other[2].view(np.int64)), name
    erp, ecol, evals, eabs = orc.spgemm_csr(A, A)
    assert_csr_close(fused[0], fused[1], fused[2], erp, ecol, evals, eabs, f"{case}: ")


@pytest.mark.parametrize("case", list(MANY_WINDOW_CASES))
def test_global_rows_atomic_adds(case, orc):
    """Heavy tile rows accumulated with atomic adds (global_rows = 2, the
    task's tables in shared memory, its entries shared by all warps): the
    structure of the shared-memory result, values within the bound of the
    oracle (the order of the adds is not fixed)."""
    A = MANY_WINDOW_CASES[case]()
    ctx = R.Context(0, dict(global_rows=2))
    got = _run(ctx, A)
    if case.startswith("rmat"):  # rows of many windows: tasks in device memory
        assert ctx.stats()["split_windows"] > 0
    ctx.close()
    ctx = R.Context(0)
    ref = _run(ctx, A)
    ctx.close()
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
    assert_csr_close(*got[:3], *orc.spgemm_csr(A, A), f"{case} global atomics: ")


def test_split_cursors_past_the_cap(orc):
    """Tile rows of 40,000 A entries (2,500 per row) against B rows of two
    scattered entries: about 40 windows per tile row, grouped 13 to a task by
    the default split target, so a worker's window cursors cover only the
    first 32,768 entries of the row and the rest take the binary search.
    Bitwise equal to the unsplit run and to the tile output, within the bar
    of the oracle."""
    rng = np.random.default_rng(81)
    m, k, n = 48, 40000, 100000
    rows = np.repeat(np.arange(m), 2500)
    cols = np.concatenate([rng.choice(k, 2500, replace=False) for _ in range(m)])
    A = G.from_coo(m, k, rows, cols, rng.uniform(-1, 1, rows.size))
    brows = np.repeat(np.arange(k), 2)
    B = G.from_coo(k, n, brows, rng.integers(0, n, brows.size), rng.uniform(-1, 1, brows.size))
    runs = {}
    for name, cfg in (("split", dict(fused_csr_output=1)),
                      ("nosplit", dict(fused_csr_output=1, split_target=-1)),
                      ("global", dict(fused_csr_output=1, global_rows=1)),
                      ("tiled", dict(fused_csr_output=0))):
        ctx = R.Context(0, cfg)
        runs[name] = _run(ctx, A, B)
        st = ctx.stats()
        if name == "split":
            assert st["split_windows"] > 0 and st["split_multi_window_tasks"] > 0, st
        ctx.close()
    ref = runs["split"]
    for name, other in runs.items():
        assert np.array_equal(ref[0], other[0]) and np.array_equal(ref[1], other[1]), name
        assert np.array_equal(ref[2].view(np.int64), other[2].view(np.int64)), name
    assert_csr_close(ref[0], ref[1], ref[2], *orc.spgemm_csr(A, B), "cursors past the cap: ")


def test_deterministic_and_reusable(orc):
    """Two runs on one context give bitwise-identical values (no atomics in
    the value accumulation), and the context can switch problems."""
    A = G.stencil_27(10, 5)
    ctx = R.Context(0)
    r1 = _run(ctx, A)
    B = G.laplacian_2d(40)
    _run(ctx, B)
    r2 = _run(ctx, A)
    assert np.array_equal(r1[0], r2[0]) and np.array_equal(r1[1], r2[1])
    assert np.array_equal(r1[2].view(np.int64), r2[2].view(np.int64))
    ctx.close()


def test_empty_and_tiny(orc):
    ctx = R.Context(0)
    for A in (G.CSR(5, 5, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0)),
              G.CSR(1, 1, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([3.0]))):
        rp, ci, va, nnz, _ = _run(ctx, A)
        erp, ecol, evals, eabs = orc.spgemm_csr(A, A)
        assert_csr_close(rp, ci, va, erp, ecol, evals, eabs, "tiny: ")
    ctx.close()


def test_host_buffer_entry(orc):
    A = G.laplacian_2d(100)
    C = R.spgemm_csr_host(A)
    erp, ecol, evals, eabs = orc.spgemm_csr(A, A)
    assert_csr_close(C.rowptr, C.col, C.val, erp, ecol, evals, eabs, "host entry: ")


def test_kat_2d_laplacian_closed_form():
    """C = A^2 of the 5-point Laplacian (diag 4, off -1) on a 256^2 grid:
    nnz(C) = 846,852; C_ii = 16 + deg(i); distance-1 entries -8; distance-2
    entries 1 (straight) or 2 (diagonal, two paths)."""
    nx = 256
    A = G.laplacian_2d(nx)
    C = R.spgemm_csr_host(A)
    assert C.nnz == 846852
    rows = np.repeat(np.arange(C.m), np.diff(C.rowptr))
    deg = np.diff(A.rowptr) - 1
    xi, yi = rows % nx, rows // nx
    xj, yj = C.col % nx, C.col // nx
    dx, dy = np.abs(xi - xj), np.abs(yi - yj)
    expect = np.where((dx == 0) & (dy == 0), 16.0 + deg[rows],
             np.where(dx + dy == 1, -8.0,
             np.where((dx == 1) & (dy == 1), 2.0, 1.0)))
    assert np.array_equal(C.val, expect)


SEGWALK_CASES = {
    "stencil27_12": lambda: G.stencil_27(12, 3),
    "lap2d_256": lambda: G.laplacian_2d(256),
    "banded": lambda: G.banded_scatter(3000, 12, seed=9),
    "ragged": lambda: G.laplacian_2d(37, 11),
    "rect": lambda: G.random_csr(300, 300, 0.02, seed=8),
}


@pytest.mark.parametrize("case", list(SEGWALK_CASES))
def test_segment_walk_equals_entry_walk(case, orc):
    """The numeric step over B's row segments (segment_walk, where it applies)
    and the entry-per-lane walk sum every output in the same order: bitwise
    the same C, and the oracle's within the bound."""
    A = SEGWALK_CASES[case]()
    got = {}
    for off in (0, 1):
        ctx = R.Context(0, dict(segment_walk=1 - off))
        rp, ci, va, nnz, _ = _run(ctx, A)
        got[off] = (rp, ci, va)
        ctx.close()
    assert np.array_equal(got[0][0], got[1][0]) and np.array_equal(got[0][1], got[1][1])
    assert np.array_equal(got[0][2].view(np.int64), got[1][2].view(np.int64))
    assert_csr_close(*got[0], *orc.spgemm_csr(A, A), f"{case} segment walk: ")


@pytest.mark.parametrize("case", ["stencil27_12", "banded", "rmat_12", "lap2d_ragged"])
def test_persistent_rows_equal_per_row_ctas(case, orc):
    """Tile-row CTAs as one resident wave over a device queue (with the split
    workers beside them for multi-window rows): bitwise the one-CTA-per-row C."""
    A = CASES[case]()
    got = {}
    for pers in (0, 1):
        ctx = R.Context(0, dict(persistent_rows=pers))
        rp, ci, va, nnz, _ = _run(ctx, A)
        got[pers] = (rp, ci, va)
        ctx.close()
    assert np.array_equal(got[0][0], got[1][0]) and np.array_equal(got[0][1], got[1][1])
    assert np.array_equal(got[0][2].view(np.int64), got[1][2].view(np.int64))
    assert_csr_close(*got[1], *orc.spgemm_csr(A, A), f"{case} persistent: ")


WIDE_WINDOW_CASES = {
    "banded": (MANY_WINDOW_CASES["banded"], R.RTT_OP_AB),
    "rmat_12_aat": (MANY_WINDOW_CASES["rmat_12"], R.RTT_OP_AAT),
    "banded_20k": (MANY_WINDOW_CASES["banded_20k"], R.RTT_OP_AB),
    "unsorted_wide": (MANY_WINDOW_CASES["unsorted_wide"], R.RTT_OP_AB),
    "rmat_14": (MANY_WINDOW_CASES["rmat_14"], R.RTT_OP_AB),
}


@pytest.mark.parametrize("case", list(WIDE_WINDOW_CASES))
def test_sym_window_slots_equal(case, orc):
    """Symbolic step 2 of tile rows with more than 254 C tiles in 254-slot
    windows (-1), in the wide-window CTAs at the default (0), the smallest
    (255) and the largest (6000) window: bitwise the same C, which matches
    the oracle."""
    make, op = WIDE_WINDOW_CASES[case]
    A = make()
    got = {}
    for slots in (-1, 0, 255, 6000):
        ctx = R.Context(0, dict(sym_window_slots=slots))
        got[slots] = _run(ctx, A, None, op)
        ctx.close()
    ref = got[-1]
    for slots, g in got.items():
        assert np.array_equal(ref[0], g[0]) and np.array_equal(ref[1], g[1]), slots
        assert np.array_equal(ref[2].view(np.int64), g[2].view(np.int64)), slots
    B = A.transpose() if op == R.RTT_OP_AAT else A
    assert_csr_close(*ref[:3], *orc.spgemm_csr(A, B), f"{case} windows: ")


def test_sym_window_slots_checked():
    for bad in (-2, 1, 254, 6001):
        with pytest.raises(R.RttError) as e:
            R.Context(0, dict(sym_window_slots=bad))
        assert e.value.status == 1  # RTT_ERR_INVALID_ARGUMENT


def test_leaf_dmma_forms(orc):
    """The leaf DMMA numeric step in the other forms: A*A^T, general A*B, a
    values-only update and a batch, each against the oracle (structure
    bit-exact, values within the bound)."""
    cfg = dict(leaf_dmma=1)
    A = G.rmat(11, 8, seed=4)
    ctx = R.Context(0, cfg)
    rp, ci, va, nnz, _ = _run(ctx, A, None, R.RTT_OP_AAT)
    assert_csr_close(rp, ci, va, *orc.spgemm_csr(A, A.transpose()), "leaf AAT: ")
    assert ctx.stats()["nnz_cub"] == orc.nnzcub(A, A.transpose())
    ctx.close()
    A2 = G.random_csr(500, 300, 0.02, seed=31)
    B2 = G.random_csr(300, 700, 0.015, seed=32)
    ctx = R.Context(0, cfg)
    rp, ci, va, nnz, _ = _run(ctx, A2, B2)
    assert_csr_close(rp, ci, va, *orc.spgemm_csr(A2, B2), "leaf A*B: ")
    ctx.close()
    # a values-only update
    S = G.stencil_27(12, 2)
    ctx = R.Context(0, cfg)
    d = torch.device("cuda:0")
    da = (S.m, S.n, torch.from_numpy(S.rowptr).to(d), torch.from_numpy(S.col).to(d),
          torch.from_numpy(S.val).to(d))
    nnz, _ = ctx.symbolic(da)
    out = (torch.empty(S.m + 1, dtype=torch.int32, device=d),
           torch.empty(nnz, dtype=torch.int32, device=d),
           torch.empty(nnz, dtype=torch.float64, device=d))
    ctx.numeric(*out)
    nv = da[4] * -0.5 + 0.25
    ctx.numeric_values(nv, None, *out)
    torch.cuda.synchronize()
    S2 = G.CSR(S.m, S.n, S.rowptr, S.col, nv.cpu().numpy())
    assert_csr_close(out[0].cpu().numpy(), out[1].cpu().numpy(), out[2].cpu().numpy(),
                     *orc.spgemm_csr(S2, S2), "leaf values-only: ")
    ctx.close()
    # a batch
    As = [G.banded_scatter(300 + 97 * i, 5, seed=i) for i in range(5)]
    ctx = R.Context(0, cfg)
    outs = R.spgemm_batched(ctx, [(X.m, X.n, torch.from_numpy(X.rowptr).to(d),
                                   torch.from_numpy(X.col).to(d), torch.from_numpy(X.val).to(d))
                                  for X in As])
    torch.cuda.synchronize()
    for X, (orp, oci, ova) in zip(As, outs):
        assert_csr_close(orp.cpu().numpy(), oci.cpu().numpy(), ova.cpu().numpy(),
                         *orc.spgemm_csr(X, X), "leaf batch: ")
    ctx.close()


def test_host_into_caller_buffers(orc):
    """rtt_spgemm_csr_host_into: C into the caller's host arrays, page-locked
    or pageable, reused across calls; too-small arrays get a clean error with
    the size, and the result equals the malloc'd-output call's bit for bit."""
    A = G.stencil_27(24, 1)  # C's values above the 4 MB of the staged copies
    ctx = R.Context(0)
    want = ctx.spgemm_csr_host(A)
    small = (np.zeros(A.m + 1, np.int32), np.zeros(10, np.int32), np.zeros(10))
    with pytest.raises(R.RttError) as e:
        ctx.spgemm_csr_host_into(A, small)
    assert e.value.status == 1 and str(want.col.size) in str(e.value)
    nnz = want.col.size
    pinned = tuple(torch.empty(n, dtype=t).pin_memory().numpy()
                   for n, t in ((A.m + 1, torch.int32), (nnz + 5, torch.int32),
                                (nnz + 5, torch.float64)))
    pageable = (np.zeros(A.m + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz))
    for out in (pinned, pageable, pinned):
        got = ctx.spgemm_csr_host_into(A, out)
        assert got == nnz
        assert np.array_equal(out[0], want.rowptr) and np.array_equal(out[1][:nnz], want.col)
        assert np.array_equal(out[2][:nnz].view(np.int64), want.val.view(np.int64))
    ctx.close()
    assert_csr_close(pageable[0], pageable[1], pageable[2], *orc.spgemm_csr(A, A), "into: ")
