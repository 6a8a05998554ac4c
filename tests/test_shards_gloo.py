"""The shard exchange of a sharded search (xtn.exchange_keys: sizes, then keys, all-to-all by
owner rank) on the CPU with gloo ranks. Each rank holds the verified pairs of its shard as
pair keys (x << (b + 8) | y << 8 | distance) sorted by (x, y), with pairs that several shards
found repeated across ranks; after the exchange and a sort-unique merge, the ranks' results in
rank order must be the whole output. The shards' contents here come from the oracle's output,
split with overlaps; the device packing and merge are tested on the GPU."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORLD = 3


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def keys_of(pairs, dist, b):
    return (pairs[:, 0].astype(np.int64) << (b + 8)) | (pairs[:, 1].astype(np.int64) << 8) | dist.astype(np.uint8)


def shard_contents(n, world, seed):
    """A sorted, unique output and, per rank, a sorted subset; every pair in at least one."""
    rng = np.random.default_rng(seed)
    x = rng.integers(0, n - 1, 4000)
    y = x + 1 + rng.integers(0, 50, 4000)
    ok = y < n
    pairs = np.unique(np.stack([x[ok], y[ok]], axis=1), axis=0).astype(np.int32)
    dist = rng.integers(0, 3, len(pairs)).astype(np.int8)
    owner = rng.integers(0, world, len(pairs))
    extra = rng.random(len(pairs)) < 0.3  # found by a second shard too
    second = (owner + 1 + rng.integers(0, world - 1, len(pairs))) % world
    shards = []
    for r in range(world):
        sel = (owner == r) | (extra & (second == r))
        shards.append((pairs[sel], dist[sel]))
    return pairs, dist, shards


def worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(ROOT, "xt-neighbor_b200"))
    import xtn

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n, b = 5000, 13
        _, _, shards = shard_contents(n, world, seed=3)
        p, d = shards[rank]
        keys = torch.from_numpy(keys_of(p, d, b))
        # owner ranges [ceil(k n / K), ceil((k + 1) n / K)) over the sorted x column
        bounds = [-(-k * n // world) for k in range(world)]
        starts = [int(np.searchsorted(p[:, 0], x0, side="left")) for x0 in bounds] + [len(p)]
        got = xtn.exchange_keys(keys, starts)
        merged = np.unique(got.numpy())
        out.put((rank, merged))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_three_rank_exchange_restores_the_output():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, WORLD, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pairs, dist, _ = shard_contents(5000, WORLD, seed=3)
    expect = keys_of(pairs, dist, 13)
    got = np.concatenate([res[r] for r in range(WORLD)])
    assert np.array_equal(got, np.sort(expect))
    for r in range(WORLD):  # each rank holds only its own id range
        x = res[r] >> (13 + 8)
        lo, hi = -(-r * 5000 // WORLD), -(-(r + 1) * 5000 // WORLD)
        assert len(x) == 0 or (x.min() >= lo and x.max() < hi)


def test_owner_ranges_cover_the_buckets_in_order():
    sys.path.insert(0, os.path.join(ROOT, "xt-neighbor_b200"))
    import xtn

    rng = np.random.default_rng(7)
    for K in (1, 2, 3, 8):
        counts = rng.integers(0, 1000, 512)
        b = xtn.owner_ranges(counts, K)
        assert b[0] == 0 and b[-1] == 512 and all(x <= y for x, y in zip(b, b[1:])) and len(b) == K + 1
        starts = np.concatenate([[0], np.cumsum(counts)])
        for k in range(1, K):  # rank k starts at the bucket holding record k V / K
            assert starts[b[k]] >= starts[-1] * k // K and (b[k] == 0 or starts[b[k] - 1] < starts[-1] * k // K)


def rank_records(r, nb=40):
    """Rank r's first-level bucket counts (some empty) and its records in bucket order, each
    encoding (source rank, bucket, index)."""
    rng = np.random.default_rng(100 + r)
    counts = rng.integers(0, 30, nb)
    counts[rng.random(nb) < 0.2] = 0
    recs = np.concatenate([[(r << 40) | (b << 20) | i for i in range(int(c))] for b, c in enumerate(counts)] +
                          [np.zeros(0, np.int64)]).astype(np.int64)
    return counts, recs


def record_worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(ROOT, "xt-neighbor_b200"))
    import xtn

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        counts, recs = rank_records(rank)
        t = torch.from_numpy(recs) if len(recs) else torch.zeros(1, dtype=torch.int64)
        got, pieces, bounds = xtn.exchange_records(counts, t)
        out.put((rank, got.numpy().copy(), pieces, bounds))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_three_rank_record_exchange_sends_each_owner_its_buckets():
    """xtn.exchange_records (the sequence-sharded search's exchange): every owner receives the
    records of its first-level buckets from every rank, one piece per source in rank order, with
    the per-bucket counts that xtn_shard_search needs to gather them."""
    sys.path.insert(0, os.path.join(ROOT, "xt-neighbor_b200"))
    import xtn

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=record_worker, args=(r, WORLD, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    res = {r: (g, pc, b) for r, g, pc, b in (q.get(timeout=120) for _ in procs)}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    data = [rank_records(r) for r in range(WORLD)]
    bounds = xtn.owner_ranges(sum(c for c, _ in data), WORLD)
    total = 0
    for k in range(WORLD):
        got, pieces, b = res[k]
        assert b == bounds
        lo, hi = bounds[k], bounds[k + 1]
        expect = np.concatenate([recs[((recs >> 20) & 0xFFFFF >= lo) & ((recs >> 20) & 0xFFFFF < hi)]
                                 for _, recs in data])
        assert np.array_equal(got, expect)
        assert pieces.shape == (WORLD, hi - lo)
        for p, (counts, _) in enumerate(data):
            assert np.array_equal(pieces[p], counts[lo:hi].astype(np.uint64))
        total += len(got)
    assert total == sum(len(r) for _, r in data)
