"""Host logic of the multi-GPU forms: one process per GPU, no data exchange.

The product shards by C tile rows: C(I, :) needs A's tile row I and all of B,
so the ranks of a row-sharded product each take a contiguous range of tile
rows of A (a CSR row block), multiply it by the full B and own that block of
C.  Nothing crosses between ranks on the data path; the blocks are only
concatenated by whoever needs all of C.  The reference has no multi-GPU path
(one GPU, one process), so this is the natural split of its work, not a
translation of a reference collective.

The benchmark's N-GPU form is replicas: every rank runs the whole product on
its own GPU and the job's throughput is all ranks' flops over the slowest
rank's time.
"""
from __future__ import annotations

import numpy as np

from .generators import CSR

TILE = 16


def row_costs(a: CSR, b: CSR) -> np.ndarray:
    """Per-row work of C = A*B: sum over the row's entries (i, k) of nnz(B(k, :))."""
    blen = np.diff(b.rowptr).astype(np.int64)
    per_entry = blen[a.col] if a.nnz else np.zeros(0, np.int64)
    csum = np.concatenate([[0], np.cumsum(per_entry)])
    return csum[a.rowptr[1:]] - csum[a.rowptr[:-1]]


def tile_row_shards(a: CSR, b: CSR, world: int) -> list[tuple[int, int]]:
    """Split A's rows into `world` contiguous blocks on tile-row boundaries,
    balancing the product work.  Returns [(row_begin, row_end)] per rank;
    blocks may be empty when there are fewer tile rows than ranks."""
    if world < 1:
        raise ValueError("world must be >= 1")
    tilem = (a.m + TILE - 1) // TILE
    cost = row_costs(a, b)
    tcost = np.add.reduceat(cost, np.arange(0, a.m, TILE)) if a.m else np.zeros(0, np.int64)
    ccum = np.concatenate([[0], np.cumsum(tcost)])
    total = ccum[-1]
    cuts = [0]
    for r in range(1, world):
        # first tile row whose prefix reaches r/world of the work
        t = int(np.searchsorted(ccum, total * r / world, side="left"))
        cuts.append(min(max(t, cuts[-1]), tilem))
    cuts.append(tilem)
    return [(min(c0 * TILE, a.m), min(c1 * TILE, a.m)) for c0, c1 in zip(cuts[:-1], cuts[1:])]


def row_block(a: CSR, r0: int, r1: int) -> CSR:
    """Rows [r0, r1) of A as a CSR of its own (same column count)."""
    e0, e1 = int(a.rowptr[r0]), int(a.rowptr[r1])
    return CSR(r1 - r0, a.n, (a.rowptr[r0:r1 + 1] - e0).astype(np.int32),
               a.col[e0:e1].copy(), a.val[e0:e1].copy())


def stitch(blocks: list[CSR], n: int) -> CSR:
    """Concatenate row blocks (in rank order) into one CSR."""
    m = sum(b.m for b in blocks)
    rp = [np.zeros(1, np.int64)]
    base = 0
    for b in blocks:
        rp.append(b.rowptr[1:].astype(np.int64) + base)
        base += int(b.rowptr[-1])
    rowptr = np.concatenate(rp)
    if base > np.iinfo(np.int32).max:
        raise OverflowError("nnz(C) exceeds int32")
    col = np.concatenate([b.col for b in blocks]) if blocks else np.zeros(0, np.int32)
    val = np.concatenate([b.val for b in blocks]) if blocks else np.zeros(0)
    return CSR(m, n, rowptr.astype(np.int32), col.astype(np.int32), val)


def max_over_ranks(x: float, group=None) -> float:
    """The slowest rank's time (all ranks call this at the same point)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def replica_throughput(world: int, flops_per_rank: float, ms_max: float) -> float:
    """Whole-job GFLOP/s of `world` replicas timed by the slowest rank."""
    return world * flops_per_rank / (ms_max * 1e-3) / 1e9
