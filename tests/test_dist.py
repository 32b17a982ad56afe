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


# ----------------------------------------------------------------------------- row-partitioned solve
def _system(N=6):
    if N == "zipf":   # random columns: every rank's halo reaches every other rank
        n = 600
        A = FB.gen_zipf(n, FB.zipf_scale(n, mean=6.0, sample=n, seed=3), seed=3)
        return A, FB.pdfiim_build(A, 0.1, 1, 1, 1, 16, "I", "B")
    A = FB.gen_convdiff3d(N, 0.5)
    F = FB.pdfiim_build(A, 0.05, 2, 2, 1)
    return A, F


def _row_sums(rp, ci, v, x):
    """CSR product, each row summed left to right with the product rounded first (the
    solve's exact-order SpMV)."""
    y = np.zeros(len(rp) - 1)
    for i in range(len(rp) - 1):
        s = 0.0
        for k in range(rp[i], rp[i + 1]):
            s = s + float(v[k]) * float(x[ci[k]])
        y[i] = s
    return y


def _keep(M, fill):
    """The triangle the solve applies to G (fill 1) and H (fill 2), as global CSR."""
    rp, ci, v = M
    orp, oci, ov = [0], [], []
    for i in range(len(rp) - 1):
        for k in range(rp[i], rp[i + 1]):
            if (fill == 1 and ci[k] < i) or (fill == 2 and ci[k] > i):
                continue
            oci.append(ci[k])
            ov.append(v[k])
        orp.append(len(oci))
    return np.array(orp), np.array(oci), np.array(ov)


def test_dist_partition_covers_rows_and_balances():
    A, F = _system(8)
    n = len(A[0]) - 1
    w = 1 + np.diff(A[0]) + np.diff(F["Gi"]) + np.diff(F["Hi"])
    for world in (1, 2, 3, 4, 7, 8, n):
        rs = FB.dist_partition(A, F, world)
        assert rs[0] == 0 and rs[-1] == n and len(rs) == world + 1
        assert (np.diff(rs) >= 1).all()
        loads = np.add.reduceat(w, rs[:-1])
        assert loads.max() <= w.sum() / world + w.max()
    with pytest.raises(FB.FiimError):
        FB.dist_partition(A, F, n + 1)


@pytest.mark.parametrize("world", [2, 3, 5])
def test_dist_plan_renumbers_monotonically(world):
    """Every rank's renumbered columns map back to the kept global columns in stored order,
    and the halo is exactly the referenced columns outside the rank's rows."""
    A, F = _system(6)
    rs = FB.dist_partition(A, F, world)
    mats = [(A, 0), ((F["Gi"], F["Gj"], F["Gv"]), 1), ((F["Hi"], F["Hj"], F["Hv"]), 2)]
    for M, fill in mats:
        Kp, Kc, _ = _keep(M, fill)
        for r in range(world):
            lo, hi = int(rs[r]), int(rs[r + 1])
            nloc = hi - lo
            p = FB.dist_plan(r, world, rs, FB.dist_rows(M, lo, hi), fill)
            nb, halo, cols = p["nbelow"], p["halo"], p["cols"]
            ext_to_global = np.concatenate([halo[:nb], np.arange(lo, hi), halo[nb:]])
            back = ext_to_global[cols]
            assert len(ext_to_global) == nb + nloc + p["nabove"]
            assert np.array_equal(p["rp"], Kp[lo:hi + 1] - Kp[lo])
            assert np.array_equal(back, Kc[Kp[lo]:Kp[hi]])
            ref = np.unique(Kc[Kp[lo]:Kp[hi]])
            ref = ref[(ref < lo) | (ref >= hi)]
            assert np.array_equal(halo, ref)
            assert (halo[:nb] < lo).all() and (halo[nb:] >= hi).all()
            if fill == 1:
                assert nb == 0     # G (upper) reaches only rows above the block
            if fill == 2:
                assert p["nabove"] == 0


def test_dist_plan_edge_cases():
    """Rows without entries, a single rank (no halo), and a block of one row."""
    n = 10
    rp = np.array([0, 2, 2, 2, 5, 5, 6, 8, 8, 9, 10], np.int32)       # rows 1, 2, 4, 7 empty
    ci = np.array([0, 9, 1, 3, 8, 5, 0, 6, 8, 9], np.int32)
    v = np.arange(10, dtype=float)
    M = (rp, ci, v)
    p = FB.dist_plan(0, 1, np.array([0, n]), FB.dist_rows(M, 0, n), 0)
    assert p["nbelow"] == 0 and p["nabove"] == 0 and len(p["halo"]) == 0
    assert np.array_equal(p["cols"], ci) and np.array_equal(p["rp"], rp)
    rs = np.array([0, 3, 4, n])
    for r in range(3):
        lo, hi = int(rs[r]), int(rs[r + 1])
        q = FB.dist_plan(r, 3, rs, FB.dist_rows(M, lo, hi), 0)
        ext = np.concatenate([q["halo"][:q["nbelow"]], np.arange(lo, hi), q["halo"][q["nbelow"]:]])
        assert np.array_equal(ext[q["cols"]], ci[rp[lo]:rp[hi]])
        assert np.array_equal(q["rp"], rp[lo:hi + 1] - rp[lo])
    with pytest.raises(FB.FiimError):
        FB.dist_plan(0, 2, np.array([0, 5, 5]), FB.dist_rows(M, 0, 5), 0)   # a rank without rows
    with pytest.raises(FB.FiimError):
        FB.dist_plan(2, 2, np.array([0, 5, n]), FB.dist_rows(M, 0, 5), 0)   # rank out of range


def _dist_rank(rank, world, port, q, which=6):
    """One rank: plan A, G, H; exchange the needs and the halo values over gloo as the
    solve does over NCCL; multiply; gather a partial dot product in rank order."""
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    A, F = _system(which)
    n = len(A[0]) - 1
    rs = FB.dist_partition(A, F, world)
    lo, hi = int(rs[rank]), int(rs[rank + 1])
    x = FB.rand_normal(n, 11)                 # every rank knows only x[lo:hi] below
    x_own = x[lo:hi].copy()
    out = {}
    for name, M, fill in (("A", A, 0), ("G", (F["Gi"], F["Gj"], F["Gv"]), 1), ("H", (F["Hi"], F["Hj"], F["Hv"]), 2)):
        Ml = FB.dist_rows(M, lo, hi)
        p = FB.dist_plan(rank, world, rs, Ml, fill)
        halo = p["halo"]
        owners = np.searchsorted(rs, halo, side="right") - 1
        # needs: what this rank asks of each owner; the owners answer with their values
        needs = [halo[owners == o].tolist() for o in range(world)]
        asked = [None] * world
        dist.all_gather_object(asked, needs)
        replies = [x_own[np.array(asked[o][rank], dtype=np.int64) - lo].tolist() if asked[o][rank] else []
                   for o in range(world)]
        answers = [None] * world
        dist.all_gather_object(answers, replies)
        vals = np.zeros(len(halo))
        for o in range(world):
            if o != rank:
                vals[owners == o] = answers[o][rank]
        nb = p["nbelow"]
        x_ext = np.concatenate([vals[:nb], x_own, vals[nb:]])
        # the kept values in stored order
        e0, e1 = int(M[0][lo]), int(M[0][hi])
        keep = [(M[1][k] >= lo + i if fill == 1 else M[1][k] <= lo + i if fill == 2 else True)
                for i in range(hi - lo) for k in range(int(M[0][lo + i]), int(M[0][lo + i + 1]))]
        v = np.asarray(M[2][e0:e1])[np.array(keep, dtype=bool)]
        y = _row_sums(p["rp"], p["cols"], v, x_ext)
        part = 0.0
        for yi in y:
            part = part + yi * yi
        parts = [None] * world
        dist.all_gather_object(parts, part)
        tot = parts[0]
        for o in range(1, world):
            tot = tot + parts[o]
        out[name] = (lo, y, tot)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out))


@pytest.mark.timeout(180)
@pytest.mark.parametrize("world,which", [(2, 6), (3, 6), (3, "zipf")])
def test_dist_halo_exchange_reproduces_global_products(world, which):
    """Ranks exchanging halos by their plans compute every row of A x, G x and H x exactly as
    the single-system product (bit for bit), and all ranks hold the same gathered sum; on a
    stencil (neighbouring ranks) and on random columns (every rank exchanges with every
    other)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dist_rank, args=(r, world, port, q, which)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=150) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    A, F = _system(which)
    n = len(A[0]) - 1
    x = FB.rand_normal(n, 11)
    for name, M, fill in (("A", A, 0), ("G", (F["Gi"], F["Gj"], F["Gv"]), 1), ("H", (F["Hi"], F["Hj"], F["Hv"]), 2)):
        ref = _row_sums(*_keep(M, fill), x)
        got = np.zeros(n)
        tots = set()
        for r in range(world):
            lo, y, tot = out[r][name]
            got[lo:lo + len(y)] = y
            tots.add(tot)
        assert np.array_equal(got, ref), name
        assert len(tots) == 1
