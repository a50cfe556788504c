"""Row-block sharding and the timing collectives on 2 CPU ranks (gloo)."""
import os
import socket

import numpy as np
import pytest

from hiperml_b200.dist import max_over_ranks, row_block


@pytest.mark.parametrize("M,world", [(65536, 8), (4096, 3), (1000, 2), (100, 4), (0, 2), (129, 2)])
def test_row_blocks_cover_rows_once(M, world):
    blocks = [row_block(M, world, r) for r in range(world)]
    assert blocks[0][0] == 0 and blocks[-1][1] == M
    for (a, b), (c, d) in zip(blocks, blocks[1:]):
        assert b == c and a <= b
    for a, b in blocks:
        assert a % 128 == 0 and (b % 128 == 0 or b == M)
    sizes = [b - a for a, b in blocks]
    assert max(sizes) - min(sizes) <= 128


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist

    import oracle
    from hiperml_b200 import datagen as dg
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        M, N, K = 700, 9, 64
        A = dg.matrix(M, K, 1, 0, order="C")
        B = dg.matrix(K, N, 1, 1, order="C")
        r0, r1 = row_block(M, world, rank)
        # each rank computes only its rows (the GPU kernel in production;
        # the oracle's loop here), B replicated: no reduction needed
        blk = oracle.sgemm_rm_f32(A[r0:r1], B)
        parts = [None] * world
        dist.all_gather_object(parts, (r0, r1, blk))
        t = max_over_ranks(10.0 + rank)
        if rank == 0:
            full = oracle.sgemm_rm_f32(A, B)
            got = np.concatenate([p[2] for p in sorted(parts, key=lambda p: p[0])])
            out.put((bool(np.array_equal(got, full)), t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_row_sharding_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in ps), [p.exitcode for p in ps]
    equal, t = q.get(timeout=10)
    assert equal
    assert t == 11.0
