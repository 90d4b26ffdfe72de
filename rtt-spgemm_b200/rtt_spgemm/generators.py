"""Seeded synthetic sparse matrices for the tiled SpGEMM workloads.

No public matrix collection is available here; these generators produce the
shapes, sizes and value distributions of the benchmark configurations:

* ``laplacian_2d``  5-point Laplacian on an nx x ny grid (diag 4, off -1).
* ``stencil_27``    27-point stencil on an nx^3 grid, off-diagonals
                    U[-1, 1) from a seed, diagonal 1 + sum |off-diagonals|.
* ``rmat``          R-MAT power-law square matrix (a, b, c, d quadrant
                    probabilities, no noise, self loops kept, duplicate edges
                    merged structurally), values U[0, 1) in CSR order from a
                    seeded splitmix64 stream.
* ``banded_scatter``  banded matrix (half-bandwidth hb, band entries kept with
                    probability p) plus U{0..smax} random off-band entries per
                    row, values U[-1, 1).
* ``brick_permutation``  symmetric 2x2x4 brick ordering of an nx^3 grid: the
                    ordering under which 16x16 tiles of the 27-point stencil
                    are dense enough for the DMMA path.

Every generator returns a :class:`CSR` with sorted, duplicate-free rows.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class CSR:
    m: int
    n: int
    rowptr: np.ndarray  # int32, m + 1
    col: np.ndarray  # int32, nnz
    val: np.ndarray  # float64, nnz

    @property
    def nnz(self) -> int:
        return int(self.col.shape[0])

    def transpose(self) -> "CSR":
        rows = np.repeat(np.arange(self.m, dtype=np.int64), np.diff(self.rowptr))
        order = np.lexsort((rows, self.col))
        counts = np.bincount(self.col, minlength=self.n)
        rp = np.zeros(self.n + 1, dtype=np.int64)
        np.cumsum(counts, out=rp[1:])
        return CSR(self.n, self.m, rp.astype(np.int32), rows[order].astype(np.int32),
                   self.val[order].copy())

    def permute_symmetric(self, perm_new_to_old: np.ndarray) -> "CSR":
        """Return P A P^T where row/column new i is old perm_new_to_old[i]."""
        old_to_new = np.empty_like(perm_new_to_old)
        old_to_new[perm_new_to_old] = np.arange(perm_new_to_old.shape[0], dtype=perm_new_to_old.dtype)
        rows = np.repeat(np.arange(self.m, dtype=np.int64), np.diff(self.rowptr))
        return from_coo(self.m, self.n, old_to_new[rows], old_to_new[self.col], self.val,
                        sum_duplicates=False)


def from_coo(m: int, n: int, rows, cols, vals, sum_duplicates: bool = True) -> CSR:
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64)
    key = rows * n + cols
    order = np.argsort(key, kind="stable")
    key = key[order]
    vals = vals[order]
    if sum_duplicates and key.size:
        uniq, start = np.unique(key, return_index=True)
        vals = np.add.reduceat(vals, start)
        key = uniq
    r = key // n
    c = key % n
    counts = np.bincount(r, minlength=m)
    rp = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(counts, out=rp[1:])
    return CSR(m, n, rp.astype(np.int32), c.astype(np.int32), vals)


def laplacian_2d(nx: int = 256, ny: int | None = None) -> CSR:
    ny = nx if ny is None else ny
    n = nx * ny
    idx = np.arange(n, dtype=np.int64)
    x = idx % nx
    y = idx // nx
    offs = [(-nx, y > 0), (-1, x > 0), (0, np.ones(n, bool)), (1, x < nx - 1), (nx, y < ny - 1)]
    cols = np.full((n, 5), -1, dtype=np.int64)
    vals = np.zeros((n, 5))
    for j, (d, ok) in enumerate(offs):
        cols[:, j] = np.where(ok, idx + d, -1)
        vals[:, j] = 4.0 if d == 0 else -1.0
    keep = cols >= 0
    counts = keep.sum(1)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rp[1:])
    return CSR(n, n, rp.astype(np.int32), cols[keep].astype(np.int32), vals[keep])


def stencil_27(nx: int = 96, seed: int = 0) -> CSR:
    n = nx ** 3
    idx = np.arange(n, dtype=np.int64)
    x = idx % nx
    y = (idx // nx) % nx
    z = idx // (nx * nx)
    cols = np.full((n, 27), -1, dtype=np.int64)
    j = 0
    for dz in (-1, 0, 1):
        okz = (z + dz >= 0) & (z + dz < nx)
        for dy in (-1, 0, 1):
            oky = okz & (y + dy >= 0) & (y + dy < nx)
            for dx in (-1, 0, 1):
                ok = oky & (x + dx >= 0) & (x + dx < nx)
                cols[:, j] = np.where(ok, idx + dx + nx * dy + nx * nx * dz, -1)
                j += 1
    keep = cols >= 0
    counts = keep.sum(1)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rp[1:])
    col = cols[keep]
    rng = np.random.default_rng(seed)
    val = rng.uniform(-1.0, 1.0, size=col.shape[0])
    row = np.repeat(idx, counts)
    diag = col == row
    val[diag] = 0.0
    absum = np.bincount(row, weights=np.abs(val), minlength=n)
    val[diag] = 1.0 + absum[row[diag]]
    return CSR(n, n, rp.astype(np.int32), col.astype(np.int32), val)


def splitmix64_unit(seed: int, count: int) -> np.ndarray:
    """U[0,1) doubles: element i is the top 53 bits of splitmix64(seed + i)."""
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) + np.arange(count, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
             + np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def rmat(scale: int = 20, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
         c: float = 0.19, seed: int = 1) -> CSR:
    n = 1 << scale
    edges = edge_factor * n
    rng = np.random.default_rng(seed)
    rows = np.zeros(edges, dtype=np.int64)
    cols = np.zeros(edges, dtype=np.int64)
    ab, abc = a + b, a + b + c
    chunk = 1 << 22
    for s in range(0, edges, chunk):
        e = min(edges, s + chunk)
        r = np.zeros(e - s, dtype=np.int64)
        cc = np.zeros(e - s, dtype=np.int64)
        for level in range(scale):
            u = rng.random(e - s)
            rb = u >= ab  # quadrants c, d: lower half
            cb = ((u >= a) & (u < ab)) | (u >= abc)  # quadrants b, d: right half
            r |= rb.astype(np.int64) << (scale - 1 - level)
            cc |= cb.astype(np.int64) << (scale - 1 - level)
        rows[s:e] = r
        cols[s:e] = cc
    key = np.unique(rows * n + cols)
    r = key // n
    cnt = np.bincount(r, minlength=n)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(cnt, out=rp[1:])
    val = splitmix64_unit(seed, key.shape[0])
    return CSR(n, n, rp.astype(np.int32), (key % n).astype(np.int32), val)


def banded_scatter(n: int, half_bw: int, p: float = 0.5, scatter_max: int = 4,
                   seed: int = 0) -> CSR:
    rng = np.random.default_rng(seed)
    offs = np.arange(-half_bw, half_bw + 1, dtype=np.int64)
    rows = np.repeat(np.arange(n, dtype=np.int64), offs.shape[0])
    cols = rows + np.tile(offs, n)
    keep = (cols >= 0) & (cols < n) & (rng.random(rows.shape[0]) < p)
    rows, cols = rows[keep], cols[keep]
    ns = rng.integers(0, scatter_max + 1, size=n)
    srow = np.repeat(np.arange(n, dtype=np.int64), ns)
    scol = rng.integers(0, n, size=srow.shape[0])
    # band keys are already sorted (row-major, offsets ascending): merge in the
    # few sorted scattered keys and drop repeats instead of sorting everything
    bkey = rows * n + cols
    skey = np.sort(srow * n + scol)
    key = np.insert(bkey, np.searchsorted(bkey, skey), skey)
    if key.size:
        key = key[np.concatenate([[True], key[1:] != key[:-1]])]
    r = key // n
    cnt = np.bincount(r, minlength=n)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(cnt, out=rp[1:])
    val = rng.uniform(-1.0, 1.0, size=key.shape[0])
    return CSR(n, n, rp.astype(np.int32), (key % n).astype(np.int32), val)


def batched_shapes(count: int, n_lo: int = 2000, n_hi: int = 200000, seed: int = 0):
    """(n_i, half-bandwidth_i) of the batched configuration's instances."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), size=count)).astype(np.int64)
    hb = rng.integers(8, 65, size=count)
    return ns, hb


def batched_instances(count: int, n_lo: int = 2000, n_hi: int = 200000, seed: int = 0,
                      which=None) -> list:
    """The batched configuration's instances: n_i log-uniform in [n_lo, n_hi],
    each banded (half-bandwidth uniform in 8..64, band entries kept with
    probability 0.5) plus 0..4 random off-band entries per row, values
    uniform in [-1, 1).  which: indices of the instances to build (all by
    default); instance i is the same matrix either way."""
    ns, hb = batched_shapes(count, n_lo, n_hi, seed)
    idx = range(count) if which is None else which
    return [banded_scatter(int(ns[i]), int(hb[i]), 0.5, 4, seed=int(seed * 100003 + i))
            for i in idx]


def random_csr(m: int, n: int, density: float, seed: int = 0, sort: bool = True,
               duplicates: float = 0.0, explicit_zeros: float = 0.0) -> CSR:
    """Uniform random CSR for edge-case tests: optionally unsorted rows,
    duplicate coordinates (fraction of entries repeated) and explicit zeros."""
    rng = np.random.default_rng(seed)
    cnt = rng.binomial(n, density, size=m) if n > 0 else np.zeros(m, dtype=np.int64)
    rows, cols = [], []
    for i in range(m):
        c = rng.choice(n, size=int(cnt[i]), replace=False) if cnt[i] else np.zeros(0, np.int64)
        if duplicates > 0 and c.size:
            extra = rng.choice(c, size=max(0, int(round(duplicates * c.size))), replace=True)
            c = np.concatenate([c, extra])
        c = np.sort(c) if sort else rng.permutation(c)
        rows.append(np.full(c.size, i, dtype=np.int64))
        cols.append(c.astype(np.int64))
    rows = np.concatenate(rows) if rows else np.zeros(0, np.int64)
    cols = np.concatenate(cols) if cols else np.zeros(0, np.int64)
    val = rng.uniform(-1.0, 1.0, size=cols.shape[0])
    if explicit_zeros > 0:
        val[rng.random(val.shape[0]) < explicit_zeros] = 0.0
    counts = np.bincount(rows, minlength=m) if m else np.zeros(0, np.int64)
    rp = np.zeros(m + 1, dtype=np.int64)
    if m:
        np.cumsum(counts, out=rp[1:])
    return CSR(m, n, rp.astype(np.int32), cols.astype(np.int32), val)


def brick_permutation(nx: int, bx: int = 2, by: int = 2, bz: int = 4) -> np.ndarray:
    """new_to_old map that numbers grid points brick by brick (x fastest inside
    a bx*by*bz brick, bricks in x-fastest order).  nx must divide by bx, by, bz."""
    assert nx % bx == 0 and nx % by == 0 and nx % bz == 0
    idx = np.arange(nx ** 3, dtype=np.int64)
    x = idx % nx
    y = (idx // nx) % nx
    z = idx // (nx * nx)
    brick = (x // bx) + (nx // bx) * ((y // by) + (nx // by) * (z // bz))
    inner = (x % bx) + bx * ((y % by) + by * (z % bz))
    key = brick * (bx * by * bz) + inner  # new index of each old point
    new_to_old = np.empty_like(idx)
    new_to_old[key] = idx
    return new_to_old
