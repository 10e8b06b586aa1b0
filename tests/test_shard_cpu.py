"""Splitting one structure's pair sums over several GPUs, on the host: the
work-item assignment of crab_shard_assign against a restatement of its rule,
and two gloo ranks that each sum their share of a tiled pair sum and
all-reduce it (the GPU run uses the same functions over NCCL)."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from crabsaxs_b200 import InvalidInput
from crabsaxs_b200 import shard as S


def _greedy(cost, n):
    load = [0] * n
    owner = []
    for c in cost:
        best = min(range(n), key=lambda s: (load[s], s))
        owner.append(best)
        load[best] += c
    return owner, load


@pytest.mark.parametrize("n_shards", [1, 2, 3, 8])
def test_shard_assign_follows_the_greedy_rule(n_shards):
    rng = np.random.default_rng(n_shards)
    cost = np.sort(rng.integers(1, 16, 500))[::-1]
    owner = S.shard_assign(cost, n_shards)
    ref, load = _greedy(cost.tolist(), n_shards)
    assert owner.tolist() == ref
    assert np.array_equal(S.shard_assign(cost, n_shards), owner)  # the same on every call (every rank)
    # longest-first greedy: no shard exceeds the mean by more than one item
    assert max(load) <= cost.sum() / n_shards + cost.max()
    assert sorted(set(owner.tolist())) == list(range(n_shards))


def test_shard_assign_edge_cases():
    assert S.shard_assign([], 4).size == 0
    assert S.shard_assign([7], 4).tolist() == [0]
    assert S.shard_assign([3, 3, 3], 5).tolist() == [0, 1, 2]  # more shards than items: the rest stay empty
    with pytest.raises(InvalidInput):
        S.shard_assign([1, 2], 0)
    with pytest.raises(InvalidInput):
        S.shard_assign([1, -2], 2)


TILE = 64


def _problem():
    rng = np.random.default_rng(11)
    xyz = rng.normal(0.0, 9.0, (300, 3))
    w = rng.uniform(1.0, 8.0, 300)
    q = np.linspace(0.0, 0.5, 17)
    return xyz, w, q


def _items(n):
    tiles = (n + TILE - 1) // TILE
    items = [(it, jt) for it in range(tiles) for jt in range(it, tiles)]
    items.sort(key=lambda p: -(2 - (p[0] == p[1])))  # longest first, stable
    return items, [2 - (it == jt) for it, jt in items]


def _pair_sum(xyz, w, q, it, jt):
    a = np.arange(it * TILE, min((it + 1) * TILE, len(w)))
    b = np.arange(jt * TILE, min((jt + 1) * TILE, len(w)))
    r = np.linalg.norm(xyz[a][:, None, :] - xyz[b][None, :, :], axis=-1)
    keep = a[:, None] < b[None, :] if it == jt else np.ones_like(r, bool)
    ww = (w[a][:, None] * w[b][None, :])[keep]
    x = q[:, None] * r[keep][None, :]
    return (ww[None, :] * np.sinc(x / np.pi)).sum(axis=1)


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    xyz, w, q = _problem()
    items, cost = _items(len(w))
    owner = S.shard_assign(cost, world)
    part = np.zeros(len(q))
    for (it, jt), o in zip(items, owner):
        if o == rank:
            part += _pair_sum(xyz, w, q, it, jt)
    total = S.reduce_shards(part)
    # the multipole moment exchange: an in-place sum of a host buffer
    moments = np.full(7, rank + 1.0)
    S._in_place_sum(None)(moments)
    dist.destroy_process_group()
    out.put((rank, int((owner == rank).sum()), total, moments))


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_sum_their_shares_to_the_whole(world):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted((out.get(timeout=180) for _ in procs), key=lambda g: g[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    xyz, w, q = _problem()
    items, _ = _items(len(w))
    whole = sum(_pair_sum(xyz, w, q, it, jt) for it, jt in items)
    # every pair i < j exactly once: at q = 0 the sum is ((Σw)² - Σw²)/2
    assert whole[0] == pytest.approx((w.sum() ** 2 - (w * w).sum()) / 2.0, rel=1e-12)
    assert sum(g[1] for g in got) == len(items) and all(g[1] > 0 for g in got)
    for _, _, total, moments in got:
        assert np.max(np.abs(total - whole)) <= 1e-12 * np.max(np.abs(whole))
        assert np.array_equal(total, got[0][2])  # every rank holds the same sum
        assert np.all(moments == world * (world + 1) / 2)


def test_reduce_without_a_process_group_is_the_identity():
    a = np.arange(6.0).reshape(2, 3)
    assert np.array_equal(S.reduce_shards(a), a)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]
