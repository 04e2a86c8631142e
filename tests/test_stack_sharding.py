"""Stack sharding across ranks (host logic; CPU only).

The multi-GPU path shards a stack by grid with no data-path collective; the
world-size-2 test runs two gloo ranks that each compute the assignment and
checks, through an all_gather, that the shares are disjoint, cover the stack
and are balanced.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from core_b200.stack import shard_stack
from core_b200.synthetic import gen_stack_meta


def test_shard_single_rank_takes_everything():
    shapes = [(10, 20), (30, 5), (7, 7)]
    assert shard_stack(shapes, 1) == [[0, 1, 2]]


def test_shard_balances_the_stack():
    meta = gen_stack_meta(64, seed=0)
    shapes = [(m[0], m[1]) for m in meta]
    for world in (2, 4, 8):
        parts = shard_stack(shapes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(shapes[i][0] * shapes[i][1] for i in p) for p in parts]
        biggest = max(h * w for h, w in shapes)
        assert max(loads) - min(loads) <= biggest


def test_shard_more_ranks_than_grids():
    parts = shard_stack([(4, 4), (5, 5)], 4)
    assert sorted(i for p in parts for i in p) == [0, 1]
    assert sum(1 for p in parts if not p) == 2


def test_shard_rejects_bad_input():
    with pytest.raises(ValueError):
        shard_stack([(1, 1)], 0)
    with pytest.raises(ValueError):
        shard_stack([(1, 1)], 2, work=[1.0, 2.0])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        meta = gen_stack_meta(64, seed=0)
        shapes = [(m[0], m[1]) for m in meta]
        mine = shard_stack(shapes, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        if rank == 0:
            q.put(got)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_a_disjoint_cover():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    a, b = map(set, got)
    assert not (a & b)
    assert a | b == set(range(64))
    meta = gen_stack_meta(64, seed=0)
    la = sum(meta[i][0] * meta[i][1] for i in a)
    lb = sum(meta[i][0] * meta[i][1] for i in b)
    assert abs(la - lb) <= max(m[0] * m[1] for m in meta)
