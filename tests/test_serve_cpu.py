"""Host logic of the serving loop that needs no GPU: the admission bound of a
request (nnzCub, C's entries bound) and the rejection of invalid operands."""
from __future__ import annotations

import numpy as np
import pytest

from rtt_spgemm import generators as G
from rtt_spgemm import serve


@pytest.mark.parametrize("op", ["A2", "AAT"])
def test_product_cub_matches_oracle(orc, op):
    A = G.banded_scatter(700, 9, seed=2)
    B = A if op == "A2" else A.transpose()
    assert serve.product_cub(A, op) == orc.nnzcub(A, B)
    assert serve.product_bound(A, op) == 12 * orc.nnzcub(A, B) + 4 * (A.m + 1)


def test_invalid_operands_rejected():
    ok = G.laplacian_2d(5)
    serve.product_cub(ok, "A2")
    bad_col = G.CSR(3, 3, np.array([0, 1, 2, 3], np.int32), np.array([0, 3, 1], np.int32),
                    np.ones(3))
    bad_ptr = G.CSR(3, 3, np.array([0, 2, 1, 3], np.int32), np.array([0, 1, 2], np.int32),
                    np.ones(3))
    rect = G.random_csr(4, 6, 0.5, seed=1)
    for a, op in ((bad_col, "A2"), (bad_ptr, "AAT"), (rect, "A2")):
        with pytest.raises(ValueError):
            serve.product_cub(a, op)
    serve.product_cub(rect, "AAT")  # A * A^T of a rectangular A is fine
