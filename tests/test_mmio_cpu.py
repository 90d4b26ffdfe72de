"""CPU: the Matrix Market reader (rtt_mmio_read) against the reference's own
mmio_allinone (src/mmio_highlevel.h:593, compiled into oracle/_ref) on
generated files - general, symmetric, hermitian, skew-symmetric, pattern,
integer and complex entries, comments and blank lines - array for array;
the value overwrite i % 10 of the reference's benchmark; and the errors the
reference does not report."""
from __future__ import annotations

import numpy as np
import pytest

import rtt_spgemm as R


def _write(path, field, symmetry, m, n, entries, comments=True, blank=False):
    lines = [f"%%MatrixMarket matrix coordinate {field} {symmetry}"]
    if comments:
        lines += ["% a comment line", "%"]
    lines.append(f"{m} {n} {len(entries)}")
    for k, (i, j, v) in enumerate(entries):
        if field == "pattern":
            lines.append(f"{i + 1} {j + 1}")
        elif field == "integer":
            lines.append(f"{i + 1} {j + 1} {int(v)}")
        elif field == "complex":
            lines.append(f"{i + 1} {j + 1} {v!r} {-v!r}")
        else:
            lines.append(f"{i + 1} {j + 1} {v!r}")
        if blank and k % 7 == 3:
            lines.append("")
    path.write_text("\n".join(lines) + "\n")
    return path


def _entries(m, n, count, seed, lower=False):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        i, j = int(rng.integers(0, m)), int(rng.integers(0, n))
        if lower and j > i:
            i, j = j, i
        out.append((i, j, float(rng.uniform(-5, 5))))
    return out


FILES = [
    ("real", "general", 40, 30, False),
    ("real", "symmetric", 50, 50, True),
    ("real", "hermitian", 20, 20, True),
    ("real", "skew-symmetric", 20, 20, True),
    ("pattern", "symmetric", 60, 60, True),
    ("pattern", "general", 10, 70, False),
    ("integer", "general", 33, 33, False),
    ("complex", "hermitian", 25, 25, True),
]


@pytest.mark.parametrize("field,symmetry,m,n,lower", FILES)
def test_mmio_matches_reference(tmp_path, ref, field, symmetry, m, n, lower):
    ents = _entries(m, n, 3 * m, seed=m + n, lower=lower)
    ents += [(i, i, 2.5) for i in range(0, min(m, n), 3)]  # diagonal entries
    ents.append(ents[0])  # a repeated coordinate stays two entries
    path = _write(tmp_path / "a.mtx", field, symmetry, m, n, ents, blank=True)
    got = R.mmio_read(path)
    rm, rn, rsym, rrp, rcol, rval = ref.mmio_allinone(path)
    assert (got.m, got.n, int(got.is_symmetric)) == (rm, rn, rsym)
    assert np.array_equal(got.rowptr, rrp)
    assert np.array_equal(got.col, rcol)
    assert np.array_equal(got.val, rval)


def test_mmio_value_overwrite(tmp_path):
    path = _write(tmp_path / "b.mtx", "real", "symmetric", 30, 30, _entries(30, 30, 80, 5, True))
    a = R.mmio_read(path, value_mode=1)
    assert np.array_equal(a.val, np.arange(a.nnz) % 10)


@pytest.mark.parametrize("text,status", [
    ("%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1.0\n", 2),     # short
    ("%%MatrixMarket matrix coordinate real general\n3 3 1\n4 1 1.0\n", 2),     # row 4 of 3
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", 1),         # not coordinate
    ("not a banner\n", 1),
])
def test_mmio_errors(tmp_path, text, status):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(R.RttError) as e:
        R.mmio_read(p)
    assert e.value.status == status


def test_mmio_missing_file(tmp_path):
    with pytest.raises(R.RttError) as e:
        R.mmio_read(tmp_path / "none.mtx")
    assert e.value.status == 1
