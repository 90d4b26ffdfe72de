"""CPU: the C-ABI library loads, exports every symbol include/rtt_spgemm.h
declares, keeps the reference SMatrix layout, and fails loudly (no CPU
fallback) when no GPU is present."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import rtt_spgemm as R
from rtt_spgemm import generators as G

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def _declared():
    names = set()
    for h in HEADERS:
        for m in re.finditer(r"^RTT_API\s+[\w\s\*]*?\b(rtt_\w+)\s*\(", h.read_text(), re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = R.lib()
    declared = _declared()
    assert declared, "no declarations parsed"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"
    assert declared <= set(R.EXPORTS) | declared


def test_python_mirror_lists_all_exports():
    assert _declared() == set(R.EXPORTS)


def test_smatrix_layout_matches_reference():
    # reference src/common.h:50-72 on LP64: 4 ints, 3 pointers, 2 ints,
    # 4 pointers, int (+pad), 6 pointers
    S = R.SMatrix
    assert C.sizeof(S) == 4 * 4 + 3 * 8 + 2 * 4 + 4 * 8 + 8 + 6 * 8
    assert S.value.offset == 16 and S.tilem.offset == 40 and S.numtile.offset == 80
    assert S.csc_tile_rowidx.offset == C.sizeof(S) - 8


def test_version_and_status_strings():
    assert b"sm_100a" in R.lib().rtt_version()
    assert R.lib().rtt_status_string(2) == b"invalid CSR"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks behaviour without a GPU")
def test_no_gpu_fails_loudly():
    A = G.laplacian_2d(8)
    with pytest.raises(R.RttError) as e:
        R.csr2tile_row_major(A)
    assert e.value.status == 7  # RTT_ERR_NO_DEVICE, no silent CPU fallback
    h = C.c_void_p()
    assert R.lib().rtt_context_create(C.byref(h), 0) == 7


def test_bad_arguments_rejected_before_device_work():
    lib = R.lib()
    assert lib.rtt_csr2tile_row_major(None) == 1
    assert lib.rtt_spgemm_tile(None, None, None) == 1
    s = R.SMatrix()
    s.m, s.n, s.nnz = 4, 4, 3  # nnz > 0 but no arrays
    assert lib.rtt_csr2tile_row_major(C.byref(s)) == 1
    a, b = R.SMatrix(), R.SMatrix()
    a.m, a.n, b.m, b.n = 4, 5, 6, 4
    assert lib.rtt_spgemm_tile(C.byref(a), C.byref(b), C.byref(R.SMatrix())) == 3
    assert lib.rtt_tile2csr(C.byref(R.SMatrix()), 12, 1) == 1  # malformed / bad tile_dim
    cfg = R.Config()
    lib.rtt_config_default(C.byref(cfg))
    assert cfg.dmma_pair_cutoff == 0 and cfg.fused_csr_output == 1  # DMMA opt-in
    assert cfg.split_target == 0  # heavy tile rows split at the default target
    assert cfg.cuda_graphs == 1  # repeated numeric phases replay a CUDA graph
    assert cfg.sym_window_slots == 0  # wide step-2 windows at their default size
    assert cfg.leaf_dmma == 0  # the scalar numeric kernel by default
    assert cfg.global_rows == 0
    assert C.sizeof(R.Config) == 14 * 4


def test_generators_shapes():
    A = G.laplacian_2d(256)
    assert (A.m, A.nnz) == (65536, 326656)
    S = G.stencil_27(10, 0)
    assert S.nnz == (3 * 10 - 2) ** 3
    rows = np.repeat(np.arange(S.m), np.diff(S.rowptr))
    diag = S.col == rows
    off = np.bincount(rows[~diag], weights=np.abs(S.val[~diag]), minlength=S.m)
    assert np.allclose(S.val[diag], 1.0 + off)
    for M in (A, S, G.rmat(10, 8, seed=1), G.banded_scatter(300, 9, seed=2)):
        assert np.all(np.diff(M.rowptr) >= 0)
        for r in range(0, M.m, max(1, M.m // 50)):
            c = M.col[M.rowptr[r]:M.rowptr[r + 1]]
            assert np.all(np.diff(c) > 0)
    p = G.brick_permutation(8)
    assert np.array_equal(np.sort(p), np.arange(512))
