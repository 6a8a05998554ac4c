"""Sharded nearest-neighbour search (context options shard_count / shard_index, one rank per
GPU on the same input): every shard searches its share of the first-level hash buckets, the
ranks exchange their verified pairs by owner (xtn_context_result_keys) and each merges what it
receives (xtn_context_merge_keys). With one GPU here, the shards run one after another in this
process and the all-to-all is done on the host with the very splits the ranks would send; the
ranks' merged results in rank order must equal the unsharded search, which the oracle pins.
The collective itself is covered on the CPU with gloo ranks (test_shards_gloo.py) and, for one
rank, over NCCL below. The sequence-sharded form (xtn_shard_generate / xtn_shard_search: every
rank generates its own sequences' records and sends them to the bucket owners) is emulated the
same way, with one context per rank."""
import numpy as np
import pytest

import oracle as orc
import xtn
from conftest import assert_same_pairs

pytestmark = pytest.mark.gpu


def sharded_on_one_gpu(torch, chars, offs, d, measure, K, **opts):
    n = len(offs) - 1
    dch = torch.from_numpy(chars).cuda()
    dof = torch.from_numpy(offs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    sent = []  # per shard: (keys on the device, range starts)
    per_shard_pairs = []
    with xtn.Context(0, **opts) as ctx:
        ctx.set_option("shard_count", K)
        for k in range(K):
            ctx.set_option("shard_index", k)
            m = ctx.nn_device(dch.data_ptr(), dof.data_ptr(), n, d, measure)
            per_shard_pairs.append(m)
            keys = torch.empty(max(m, 1), dtype=torch.int64, device="cuda")
            starts = ctx.result_keys(n, keys.data_ptr(), keys.numel(), K)
            assert starts[0] == 0 and starts[K] == m and all(a <= b for a, b in zip(starts, starts[1:]))
            sent.append((keys, starts))
    pairs, dists = [], []
    with xtn.Context(0) as merger:
        for dst in range(K):
            recv = [keys[starts[dst]: starts[dst + 1]] for keys, starts in sent]
            got = torch.cat(recv) if recv else torch.empty(0, dtype=torch.int64, device="cuda")
            u = merger.merge_keys(n, got.data_ptr(), got.numel())
            r = merger.fetch(u)
            lo, hi = -(-dst * n // K), -(-(dst + 1) * n // K)
            assert u == 0 or (r.pairs[:, 0].min() >= lo and r.pairs[:, 0].max() < hi), "pair outside the owner's range"
            pairs.append(r.pairs)
            dists.append(r.distances)
    return np.concatenate(pairs), np.concatenate(dists), per_shard_pairs


@pytest.mark.parametrize("kind,n,d,measure,K", [("clusters", 60_000, 2, 0, 2), ("clusters", 60_000, 2, 0, 3),
                                                ("clusters", 60_000, 2, 1, 8), ("mutants", 10_000, 1, 0, 4),
                                                ("mutants", 8_000, 3, 0, 2)])
def test_sharded_search_equals_oracle(kind, n, d, measure, K):
    import torch

    chars, offs = (xtn.synth_clusters(seed=17, n=n) if kind == "clusters" else xtn.synth_mutants(seed=19, n=n))
    exp_p, exp_d, _ = orc.nn_search(chars, offs, d, measure)
    got_p, got_d, per_shard = sharded_on_one_gpu(torch, chars, offs, d, measure, K)
    assert_same_pairs(got_p, got_d, exp_p, exp_d, f"{K} shards")
    assert sum(per_shard) >= len(exp_p)  # a pair may be found by several shards, never by none


def test_more_shards_than_buckets_and_small_rounds():
    """Shards that own no first-level bucket return nothing; a shard that needs several rounds
    under a small round limit still returns its exact share."""
    import torch

    chars, offs = xtn.synth_mutants(seed=23, n=3_000)
    exp_p, exp_d, _ = orc.nn_search(chars, offs, 1, 0)
    got_p, got_d, per_shard = sharded_on_one_gpu(torch, chars, offs, 1, 0, 64)
    assert_same_pairs(got_p, got_d, exp_p, exp_d, "64 shards")
    assert min(per_shard) == 0
    chars, offs = xtn.synth_clusters(seed=29, n=40_000)
    exp_p, exp_d, _ = orc.nn_search(chars, offs, 2, 0)
    got_p, got_d, _ = sharded_on_one_gpu(torch, chars, offs, 2, 0, 3, max_round_records=200_000)
    assert_same_pairs(got_p, got_d, exp_p, exp_d, "3 shards in rounds")


def test_shard_options_are_checked():
    import torch

    chars, offs = xtn.synth_mutants(seed=31, n=2_000)
    dch = torch.from_numpy(chars).cuda()
    dof = torch.from_numpy(offs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    with xtn.Context(0) as ctx:
        ctx.set_option("shard_count", 2)
        ctx.set_option("shard_index", 2)
        with pytest.raises(xtn.XtnError, match="shard_index must be below shard_count"):
            ctx.nn_device(dch.data_ptr(), dof.data_ptr(), 2000, 1, 0)
        ctx.set_option("shard_index", 0)
        ctx.set_option("engine", 1)
        with pytest.raises(xtn.XtnError, match="sharding needs the bucket engine"):
            ctx.nn_device(dch.data_ptr(), dof.data_ptr(), 2000, 1, 0)
        ctx.set_option("engine", 0)
        info = np.stack([np.ones(2000), np.zeros(2000), np.arange(2000)], axis=1).astype(np.int32)
        with pytest.raises(xtn.XtnError, match="nearest-neighbour mode only"):
            ctx.perform(chars, offs, distance=1, info=info, n_reps=1)


def test_nn_sharded_over_nccl_one_rank():
    """xtn.nn_sharded end to end through torch.distributed over NCCL (one rank on the one GPU):
    the all-to-all plumbing runs and the result is the whole search."""
    import datetime
    import os
    import socket

    import torch
    import torch.distributed as dist

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        chars, offs = xtn.synth_clusters(seed=37, n=30_000)
        exp_p, exp_d, _ = orc.nn_search(chars, offs, 2, 0)
        dch = torch.from_numpy(chars).cuda()
        dof = torch.from_numpy(offs.view(np.int32)).cuda()
        torch.cuda.synchronize()
        with xtn.Context(0) as ctx:
            u = xtn.nn_sharded(ctx, dch.data_ptr(), dof.data_ptr(), 30_000, 2, 0)
            r = ctx.fetch(u)
        assert_same_pairs(r.pairs, r.distances, exp_p, exp_d, "nn_sharded, one rank")
    finally:
        dist.destroy_process_group()


def exchange_on_one_gpu(torch, chars, offs, d, measure, K):
    """The sequence-sharded search (xtn_shard_generate / xtn_shard_search) with its K ranks run
    one after another on the one GPU; the two all-to-alls (records by bucket owner, then
    verified pairs by id owner) are done on the device with the very splits the ranks would
    send."""
    n = len(offs) - 1
    dch = torch.from_numpy(chars).cuda()
    dof = torch.from_numpy(offs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    ctxs = [xtn.Context(0) for _ in range(K)]
    try:
        gen = []
        for r in range(K):
            counts, ptr, nrec = ctxs[r].shard_generate(dch.data_ptr(), dof.data_ptr(), n, d, measure, r, K)
            recs = torch.as_tensor(xtn._DeviceWords(ptr, nrec), device="cuda") if nrec else None
            gen.append((counts.astype(np.int64), recs))
        nb = len(gen[0][0])
        assert all(len(c) == nb for c, _ in gen), "every rank must derive the same first-level buckets"
        total = sum(c for c, _ in gen)
        assert int(total.sum()) == int(sum(0 if r is None else r.numel() for _, r in gen))
        bounds = xtn.owner_ranges(total, K)
        received = []
        for k in range(K):
            lo, hi = bounds[k], bounds[k + 1]
            parts, pcs = [], []
            for counts, recs in gen:
                cum = np.concatenate([[0], np.cumsum(counts)])
                if recs is not None and cum[hi] > cum[lo]:
                    parts.append(recs[int(cum[lo]): int(cum[hi])].clone())
                pcs.append(counts[lo:hi])
            got = torch.cat(parts) if parts else torch.zeros(1, dtype=torch.int64, device="cuda")
            received.append((got, np.stack(pcs).astype(np.uint64)))
        torch.cuda.synchronize()
        sent = []
        for k in range(K):
            got, pcs = received[k]
            m = ctxs[k].shard_search(dch.data_ptr(), dof.data_ptr(), n, d, measure, got.data_ptr(), pcs)
            keys = torch.empty(max(m, 1), dtype=torch.int64, device="cuda")
            starts = ctxs[k].result_keys(n, keys.data_ptr(), keys.numel(), K)
            sent.append((keys, starts))
        pairs, dists = [], []
        for dst in range(K):
            got = torch.cat([keys[st[dst]: st[dst + 1]] for keys, st in sent])
            u = ctxs[dst].merge_keys(n, got.data_ptr(), got.numel())
            r = ctxs[dst].fetch(u)
            pairs.append(r.pairs)
            dists.append(r.distances)
        return np.concatenate(pairs), np.concatenate(dists)
    finally:
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("kind,n,d,measure,K", [("clusters", 60_000, 2, 0, 2), ("clusters", 60_000, 2, 1, 3),
                                                ("clusters", 60_000, 2, 0, 8), ("mutants", 10_000, 1, 0, 4),
                                                ("mutants", 3_000, 2, 0, 64)])
def test_exchange_sharded_search_equals_oracle(kind, n, d, measure, K):
    import torch

    chars, offs = (xtn.synth_clusters(seed=41, n=n) if kind == "clusters" else xtn.synth_mutants(seed=43, n=n))
    exp_p, exp_d, _ = orc.nn_search(chars, offs, d, measure)
    got_p, got_d = exchange_on_one_gpu(torch, chars, offs, d, measure, K)
    assert_same_pairs(got_p, got_d, exp_p, exp_d, f"{K} ranks with the record exchange")


def test_exchange_sharding_checks_its_inputs():
    import torch

    chars, offs = xtn.synth_mutants(seed=47, n=2_000)
    dch = torch.from_numpy(chars).cuda()
    dof = torch.from_numpy(offs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    with xtn.Context(0) as ctx:
        with pytest.raises(xtn.XtnError, match="distance <= 2"):
            ctx.shard_generate(dch.data_ptr(), dof.data_ptr(), 2000, 3, 0, 0, 2)
        with pytest.raises(xtn.XtnError, match="invalid arguments"):
            ctx.shard_generate(dch.data_ptr(), dof.data_ptr(), 2000, 1, 0, 2, 2)
        bad = offs.copy()
        bad[11] = bad[10]
        dof.copy_(torch.from_numpy(bad.view(np.int32)).cuda())
        torch.cuda.synchronize()
        with pytest.raises(xtn.XtnError, match="sequence 10 has an invalid length"):
            ctx.shard_generate(dch.data_ptr(), dof.data_ptr(), 2000, 1, 0, 0, 2)


def test_nn_sharded_exchange_over_nccl_one_rank():
    """xtn.nn_sharded_exchange end to end through torch.distributed over NCCL (one rank)."""
    import datetime
    import os
    import socket

    import torch
    import torch.distributed as dist

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        chars, offs = xtn.synth_clusters(seed=53, n=30_000)
        exp_p, exp_d, _ = orc.nn_search(chars, offs, 2, 0)
        dch = torch.from_numpy(chars).cuda()
        dof = torch.from_numpy(offs.view(np.int32)).cuda()
        torch.cuda.synchronize()
        with xtn.Context(0) as ctx:
            u = xtn.nn_sharded_exchange(ctx, dch.data_ptr(), dof.data_ptr(), 30_000, 2, 0)
            r = ctx.fetch(u)
        assert_same_pairs(r.pairs, r.distances, exp_p, exp_d, "nn_sharded_exchange, one rank")
    finally:
        dist.destroy_process_group()
