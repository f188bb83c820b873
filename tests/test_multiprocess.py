"""Two ranks over the gloo backend on CPU: the protocol of target shards.

Each rank evaluates one shard of the same particles (FMM.set_shard on a GPU; here the oracle's FP64 FMM, with
the Lagrange kernel, stands in for the evaluation and shard_indices selects the shard's particles), leaves the other particles at zero,
and an all-reduce (sum) of the ranks' results gives the whole evaluation.  Also the max-over-ranks reduction
of the step times that bench.py uses for N > 1."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O
import scalfmm_b200 as S

CENTER = (0.5, 0.5, 0.5)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shard_rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        n, order, height = 1500, 4, 4
        x, y, z = rng.random((3, n))
        q = rng.uniform(-1.0, 1.0, n)
        whole = O.fmm(O.LAGRANGE, order, height, 1.0, CENTER, x, y, z, q)
        mine = S.shard_indices(x, y, z, height, rank, world)
        part = {}
        for k in ("phi", "fx", "fy", "fz"):
            v = np.zeros(n)
            v[mine] = whole[k][mine]
            t = torch.from_numpy(v)
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
            part[k] = t.numpy()
        owned = torch.zeros(n, dtype=torch.int64)
        owned[torch.from_numpy(mine)] = 1
        dist.all_reduce(owned, op=dist.ReduceOp.SUM)
        # the step-time reduction of bench.py: every rank holds the slowest rank's times
        t = torch.tensor([1.0 + rank, 2.0 - rank], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out.put((rank, len(mine), bool((owned == 1).all()),
                 max(S.rel_l2(part[k], whole[k]) for k in part), t.tolist()))
    finally:
        dist.destroy_process_group()


def test_shards_over_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = []
    for p in procs:
        p.join(timeout=180)
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0
    res = [out.get(timeout=10) for _ in range(world)]
    res.sort()
    sizes = [r[1] for r in res]
    assert sum(sizes) == 1500 and min(sizes) > 0
    for rank, size, covered_once, err, times in res:
        assert covered_once, rank
        assert err == 0.0, (rank, err)
        assert times == [2.0, 2.0], times


@pytest.mark.parametrize("count", [1, 2, 3, 7])
def test_shard_indices_partition(count):
    """shard_indices cuts the particles into disjoint, covering, whole-leaf ranges of about N / count."""
    rng = np.random.default_rng(7)
    n = 5000
    x, y, z = rng.random((3, n))
    parts = [S.shard_indices(x, y, z, 5, r, count) for r in range(count)]
    allidx = np.sort(np.concatenate(parts))
    assert np.array_equal(allidx, np.arange(n))
    side = 16
    leaf = (np.minimum((x * side).astype(int), 15) * side + np.minimum((y * side).astype(int), 15)) * side + \
        np.minimum((z * side).astype(int), 15)
    for p in parts:
        assert abs(p.size - n / count) <= 2 * np.bincount(leaf).max()
    # whole leaves: no leaf is split between two shards
    owner = np.empty(n, np.int64)
    for r, p in enumerate(parts):
        owner[p] = r
    for l in np.unique(leaf):
        assert np.unique(owner[leaf == l]).size == 1
