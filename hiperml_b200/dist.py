"""Multi-GPU plumbing of the skinny path: one process per GPU.

The path shards by row blocks: a tall-skinny C = A B splits into contiguous
blocks of rows of A (and C), B is replicated (one broadcast), and each rank
computes its block with no data-path collective and no reduction.  The only
collectives are the timing ones: a barrier around the timed region and the
maximum of the per-rank device times.
"""
from __future__ import annotations


def row_block(M: int, world: int, rank: int, align: int = 128):
    """[start, stop) of `rank`'s rows when M rows are cut into `world`
    contiguous blocks whose boundaries fall on multiples of `align` (one SIMT
    or tensor-core tile), sizes as even as that allows."""
    if world < 1 or not 0 <= rank < world or M < 0 or align < 1:
        raise ValueError("bad partition arguments")
    tiles = (M + align - 1) // align
    lo = tiles * rank // world
    hi = tiles * (rank + 1) // world
    return min(M, lo * align), min(M, hi * align)


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank float over the default process group (the value
    itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
