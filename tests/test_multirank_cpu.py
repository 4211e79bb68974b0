"""The multi-GPU split on CPU: two gloo ranks each enumerate their contiguous rank range with the
oracle (standing in for one GPU each), gather their objective levels and merge them; the merge must
equal one exhaustive enumeration (the same shard/merge code bench.py uses on GPUs)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import cases
import oracle
import sqsgenerator_b200 as S
from sqsgenerator_b200.shard import merge_levels, shard_range


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, keep, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = S.parse_config(cases.fcc32("double", composition={"Ti": 5, "Al": 27}, iteration_mode="systematic",
                                       seed=None, iterations=None, keep=keep, pair_weights=None))
        d = S.prepare(c)
        first, count = shard_range(c.iterations, world, rank)
        mine = oracle.systematic_levels(d[0], keep=keep, threads=1, first=first, count=count)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        if rank == 0:
            out.put((c.iterations, merge_levels(gathered, keep), oracle.systematic_levels(d[0], keep=keep, threads=2)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("keep", [1, 5])
def test_two_rank_split_merges_to_the_whole(keep):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, keep, q)) for r in range(2)]
    for p in procs:
        p.start()
    total, merged, whole = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert total == 201376  # C(32, 5)
    assert merged == whole


def test_shard_range_covers_everything_once():
    for total in (0, 1, 7, 601080390):
        for world in (1, 2, 3, 8):
            spans = [shard_range(total, world, r) for r in range(world)]
            assert sum(c for _, c in spans) == total
            assert all(spans[r][0] + spans[r][1] == spans[r + 1][0] for r in range(world - 1))
