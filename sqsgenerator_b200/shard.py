"""Splitting one job across GPUs and merging the shares' objective levels.

The configuration space of a job (random: configuration indices; systematic: ranks) is cut into
contiguous ranges, one per process, like optimizer_base::iteration_range (include/sqsgen/sqs.h:226-238):
an even split with the remainder going to the lowest ranks. Each process runs its range with
sqsg_job.range_first / range_count; the ranges' objective levels combine exactly because counts add
and the two checksum halves are sums mod 2^32.
"""
from __future__ import annotations


def shard_range(total: int, world: int, rank: int) -> tuple[int, int]:
    """(first, count) of `rank`'s share of `total` configurations."""
    share, rem = divmod(total, world)
    first = rank * share + min(rank, rem)
    return first, share + (1 if rank < rem else 0)


def merge_levels(level_lists, keep: int):
    """Merge per-share levels [(objective, count, checksum)] into the keep+1 best overall."""
    merged: dict = {}
    for levels in level_lists:
        for value, count, checksum in levels:
            acc = merged.setdefault(value, [0, 0, 0])
            acc[0] += count
            acc[1] = (acc[1] + (checksum & 0xFFFFFFFF)) & 0xFFFFFFFF
            acc[2] = (acc[2] + (checksum >> 32)) & 0xFFFFFFFF
    out = [(v, a[0], a[1] | (a[2] << 32)) for v, a in sorted(merged.items())]
    return out[: keep + 1]
