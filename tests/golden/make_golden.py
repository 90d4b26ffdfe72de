"""Generate the golden fixtures in this directory from the reference's own CPU
code (oracle/_ref, compiled unmodified from the reference sources).

Each fixture stores a small input CSR and the reference's outputs of
csr2tile_row_major, csr2tile_col_major and spgemm_cpu (with the in-tile column
fix applied at the call site).  Run from the repository root:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "rtt-spgemm_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

import oracle  # noqa: E402
from rtt_spgemm import generators as G  # noqa: E402

CASES = {
    "lap2d_16": (lambda: G.laplacian_2d(16), True),
    "lap2d_ragged_13x7": (lambda: G.laplacian_2d(13, 7), True),
    "random_unsorted_48": (lambda: G.random_csr(48, 48, 0.12, seed=3, sort=False), True),
    "random_duplicates_40": (lambda: G.random_csr(40, 40, 0.15, seed=4, duplicates=0.3), True),
    "random_rect_37x53": (lambda: G.random_csr(37, 53, 0.1, seed=2), None),
    "stencil27_4": (lambda: G.stencil_27(4, 1), True),
}

ROW = ["tile_ptr", "tile_columnidx", "tile_rowidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col",
       "tile_csr_Value", "mask"]
COL = ROW + ["csc_tile_ptr", "csc_tile_rowidx"]


def main() -> None:
    oracle.build(reference=True)
    ref = oracle.Reference()
    for name, (make, square) in CASES.items():
        A = make()
        rm = ref.csr2tile_row_major(A)
        cm = ref.csr2tile_col_major(A)
        out = dict(m=A.m, n=A.n, rowptr=A.rowptr, col=A.col, val=A.val)
        out.update({"row_" + k: rm[k] for k in ROW})
        out.update({"col_" + k: cm[k] for k in COL})
        if square:
            c = ref.spgemm_cpu(rm, cm)
            out.update({"c_" + k: c[k] for k in ("tile_ptr", "tile_columnidx", "tile_nnz",
                                                  "tile_csr_Ptr", "tile_csr_Col",
                                                  "tile_csr_Value")})
            # spgemm_cpu keeps its step-3 row-length quirk (visible only on ragged n)
            out["quirk"] = np.array(1)
        np.savez_compressed(Path(__file__).resolve().parent / f"{name}.npz", **out)
        print("wrote", name)


if __name__ == "__main__":
    main()
