"""Host logic of the multi-GPU forms, run as world-size-2 gloo process groups
on the CPU (127.0.0.1).  The GPU work of each rank is stood in for by the
oracle's row product, which is what a rank's block of C must equal."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

import oracle as O
from rtt_spgemm import generators as G
from rtt_spgemm import shards

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_tile_row_shards_cover_and_align(world):
    A = G.stencil_27(6, 1)  # 216 rows, 14 tile rows (last one partial)
    sh = shards.tile_row_shards(A, A, world)
    assert len(sh) == world
    assert sh[0][0] == 0 and sh[-1][1] == A.m
    for (r0, r1), (s0, _) in zip(sh, sh[1:]):
        assert r1 == s0 and r0 <= r1
    assert all(r0 % 16 == 0 for r0, _ in sh)
    cost = shards.row_costs(A, A)
    assert cost.sum() == O.Oracle().nnzcub(A, A)


def test_stitch_roundtrip(orc):
    A = G.random_csr(300, 200, 0.03, seed=5)
    blocks = [shards.row_block(A, r0, r1) for r0, r1 in shards.tile_row_shards(A, A.transpose(), 4)]
    S = shards.stitch(blocks, A.n)
    assert np.array_equal(S.rowptr, A.rowptr) and np.array_equal(S.col, A.col)
    assert np.array_equal(S.val, A.val)


def _rank(rank: int, world: int, port: int, case: str):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        orc = O.Oracle()
        A = G.stencil_27(8, 3) if case == "stencil" else G.rmat(9, 8, seed=2)
        r0, r1 = shards.tile_row_shards(A, A, world)[rank]
        blk = shards.row_block(A, r0, r1)
        rp, col, val, _ = orc.spgemm_csr(blk, A)  # this rank's block of C = A * A
        mine = G.CSR(blk.m, A.n, rp.astype(np.int32), col, val)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        # replica timing: every rank reports its own time, the job takes the max
        t = shards.max_over_ranks(1.0 + rank)
        assert t == float(world)
        assert shards.replica_throughput(world, 2e9, t) == pytest.approx(world * 2e9 / (t * 1e-3) / 1e9)
        if rank == 0:
            C = shards.stitch(gathered, A.n)
            erp, ecol, evals, _ = orc.spgemm_csr(A, A)
            assert np.array_equal(C.rowptr.astype(np.int64), erp.astype(np.int64))
            assert np.array_equal(C.col, ecol)
            assert np.array_equal(C.val.view(np.int64), evals.view(np.int64))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["stencil", "rmat"])
def test_row_sharded_product_world2(case):
    """Two gloo ranks each multiply their tile-row block of A by A; the
    stitched blocks equal the single-process product bit for bit."""
    mp.spawn(_rank, args=(2, _free_port(), case), nprocs=2, join=True)
