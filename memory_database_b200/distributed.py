"""Row-sharded star-join over several ranks (one process per GPU).

Fact rows are independent, so each rank scans its own contiguous shard with
the dimension vectors replicated on every rank, and the only exchange of the
distributed query is one sum all-reduce of the int64 group vector (NCCL over
NVLink between GPUs; any torch.distributed backend works, the tests use
gloo on CPU).  No collective runs inside the scan.
"""
from __future__ import annotations


def shard_range(n_rows: int, rank: int, world: int) -> tuple[int, int]:
    """Rows [begin, end) of `rank`: contiguous, sizes differing by at most 1."""
    if world < 1 or not 0 <= rank < world or n_rows < 0:
        raise ValueError("bad shard arguments")
    base, rem = divmod(n_rows, world)
    begin = rank * base + min(rank, rem)
    return begin, begin + base + (1 if rank < rem else 0)


def reduce_group_sums(group_sums, group=None):
    """The exchange step: sum the ranks' int64 group vectors in place."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(group_sums, op=dist.ReduceOp.SUM, group=group)
    return group_sums


def sharded_starjoin(dimvecs, fks, factors, m1, m2, group_nums: int, aggs, ctx=None, group=None,
                     dimvec_lens=None, out=None, totals_out=None):
    """Star-join of this rank's shard of a fact table that every rank holds
    whole (device tensors), followed by the all-reduce; every rank ends with
    the group sums and totals of the whole table."""
    import torch.distributed as dist
    from .olapcore import starjoin_groupsum
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    n = int(fks[0].numel()) if len(fks) else int(m1.numel())
    b, e = shard_range(n, rank, world)
    gs, tot = starjoin_groupsum(dimvecs, fks, factors, m1, m2, group_nums, aggs=aggs, row_range=(b, e),
                                dimvec_lens=dimvec_lens, ctx=ctx, out=out, totals_out=totals_out)
    reduce_group_sums(gs, group)
    reduce_group_sums(tot, group)
    return gs, tot
