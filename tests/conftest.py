"""Shared test set-up: import paths, the gpu marker, oracle fixtures, checks."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
for sub in ("rtt-spgemm_b200", "oracle"):
    p = str(ROOT / sub)
    if p not in sys.path:
        sys.path.insert(0, p)

import oracle as _oracle  # noqa: E402

# Value tolerance of the product: |dC_ij| <= VALUE_RTOL * (|A||B|)_ij.
VALUE_RTOL = 1e-12


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    return _oracle.Oracle()


@pytest.fixture(scope="session")
def ref():
    if not _oracle.reference_available():
        pytest.skip("reference CPU code not built (oracle/_ref)")
    return _oracle.Reference()


def assert_tiles_equal(got: dict, want: dict, keys, tag: str = ""):
    for k in keys:
        g, w = got[k], want[k]
        if isinstance(w, np.ndarray):
            assert g.shape == w.shape, f"{tag}{k}: shape {g.shape} != {w.shape}"
            if not np.array_equal(g, w):
                bad = np.nonzero(g != w)[0][:5]
                raise AssertionError(f"{tag}{k}: differs at {bad}: got {g[bad]} want {w[bad]}")
        else:
            assert g == w, f"{tag}{k}: {g} != {w}"


def assert_csr_close(rowptr, col, val, want_rp, want_col, want_val, want_abs, tag: str = ""):
    """Structure bit-exact; values within VALUE_RTOL * (|A||B|)_ij."""
    rowptr = np.asarray(rowptr, dtype=np.int64)
    assert np.array_equal(rowptr, np.asarray(want_rp, dtype=np.int64)), f"{tag}row pointer differs"
    assert np.array_equal(np.asarray(col), np.asarray(want_col)), f"{tag}column indices differ"
    err = np.abs(np.asarray(val) - want_val)
    lim = VALUE_RTOL * want_abs
    ok = err <= lim
    assert ok.all(), (f"{tag}value error above {VALUE_RTOL}*|A||B|: max err {err.max():.3e}, "
                      f"worst ratio {(err / np.maximum(want_abs, 1e-300)).max():.3e}")
    return float(err.max()) if err.size else 0.0
