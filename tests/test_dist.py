"""Multi-rank host logic on CPU (gloo, world size 2): the sharding of independent units
(batched systems, right-hand sides) and the max-over-ranks timing the bench uses. No GPU:
the ranks exchange only host tensors."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import fiim_b200 as FB


def test_shard_by_nnz_covers_every_unit_once():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 4, 8):
        w = rng.integers(1000, 70000, size=256)
        shards = [FB.shard_by_nnz(w, world, r) for r in range(world)]
        assert shards[0][0] == 0 and shards[-1][1] == len(w)
        for (a, b), (c, d) in zip(shards, shards[1:]):
            assert b == c and a <= b
        loads = [w[a:b].sum() for a, b in shards]
        assert max(loads) <= w.sum() / world + w.max()        # balanced within one unit
    assert FB.shard_by_nnz([5], 2, 1) in ((1, 1), (0, 1))


def test_rhs_shards_are_contiguous_and_even():
    """The multi-RHS leg gives each rank a contiguous share of the 32 right-hand sides."""
    for world in (1, 2, 4, 8):
        shards = [FB.shard_by_nnz([1] * 32, world, r) for r in range(world)]
        assert shards[0][0] == 0 and shards[-1][1] == 32
        assert all(b == c for (_, b), (c, _) in zip(shards, shards[1:]))
        assert {b - a for a, b in shards} == {32 // world}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sides = [FB.batch_params(20261203, k)[0] for k in range(256)]
    lo, hi = FB.shard_by_nnz([5 * s * s for s in sides], world, rank)
    # every rank reports its shard; the union must be all systems, each once
    got = [None] * world
    dist.all_gather_object(got, (lo, hi))
    # max-over-ranks of a per-rank "time", as bench.py takes it
    t = torch.tensor([float(10 + rank)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got, float(t.item())))


@pytest.mark.timeout(120)
def test_two_rank_sharding_and_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=100) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, got, tmax in out:
        assert tmax == 11.0
        assert got[0][0] == 0 and got[0][1] == got[1][0] and got[1][1] == 256
