"""Resident deletion index (xtn_index_*): query batches against an index must return exactly the
pairs that the offline search reports on (index sequences followed by the batch) with one
side in the index and the other in the batch. The same holds for every request of the serving
loop, including requests split into pieces by the batch budget.
"""
import numpy as np
import pytest

import oracle as orc
import xtn
from conftest import csr

pytestmark = pytest.mark.gpu

ALPHA = "ACDEFGHIKLMNPQRSTVWY"


def seqs_of(chars, offs):
    b = chars.tobytes()
    return [b[offs[i] : offs[i + 1]].decode() for i in range(len(offs) - 1)]


def mutate(s, rng, k):
    s = list(s)
    for _ in range(k):
        op = rng.integers(3)
        p = int(rng.integers(len(s)))
        if op == 0:
            s[p] = ALPHA[int(rng.integers(20))]
        elif op == 1:
            s.insert(p, ALPHA[int(rng.integers(20))])
        elif len(s) > 1:
            del s[p]
    return "".join(s)


def make_queries(index_seqs, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        base = index_seqs[int(rng.integers(len(index_seqs)))]
        kind = i % 4
        if kind == 0:
            out.append(base)  # exact copy: distance 0
        elif kind == 3:
            out.append("".join(rng.choice(list(ALPHA), int(rng.integers(8, 23)))))
        else:
            out.append(mutate(base, rng, kind))
    return out


def offline_cross(index_seqs, query_seqs, d, measure):
    """The offline GPU search on the union, restricted to (index row, batch row) pairs."""
    chars, offs = csr(index_seqs + query_seqs)
    ctx = xtn.Context(0)
    r = ctx.perform(chars, offs, distance=d, measure=measure)
    ctx.close()
    n = len(index_seqs)
    sel = (r.pairs[:, 0] < n) & (r.pairs[:, 1] >= n)
    return r.pairs[sel], r.distances[sel]


@pytest.fixture(scope="module")
def index_setup():
    chars, offs = xtn.synth_clusters(321, 100_000, 0.20, 0.02)
    index_seqs = seqs_of(chars, offs)
    ix = xtn.Index(chars, offs, max_distance=2)
    yield ix, index_seqs
    ix.close()


@pytest.mark.parametrize("d,measure", [(1, 0), (2, 0), (1, 1), (2, 1)])
def test_query_equals_offline_union(index_setup, d, measure):
    ix, index_seqs = index_setup
    q = make_queries(index_seqs, 3000, seed=d * 10 + measure)
    qc, qo = csr(q)
    got = ix.query(qc, qo, distance=d, measure=measure)
    exp_p, exp_d = offline_cross(index_seqs, q, d, measure)
    assert len(exp_p) > 500
    assert np.array_equal(got.pairs, exp_p)
    assert np.array_equal(got.distances, exp_d)


def test_query_equals_oracle_small():
    """Against the CPU oracle itself on a union small enough for it."""
    chars, offs = xtn.synth_clusters(77, 20_000, 0.30, 0.02)
    index_seqs = seqs_of(chars, offs)
    q = make_queries(index_seqs, 800, seed=5)
    with xtn.Index(chars, offs, max_distance=2) as ix:
        for d in (1, 2):
            got = ix.query(*csr(q), distance=d)
            uc, uo = csr(index_seqs + q)
            p, dist, _ = orc.nn_search(uc, uo, d, 0)
            sel = (p[:, 0] < len(index_seqs)) & (p[:, 1] >= len(index_seqs))
            assert np.array_equal(got.pairs, p[sel])
            assert np.array_equal(got.distances, dist[sel])


def test_device_query_and_limits(index_setup):
    import torch

    ix, index_seqs = index_setup
    q = make_queries(index_seqs, 500, seed=9)
    qc, qo = csr(q)
    host = ix.query(qc, qo, distance=2)
    dch = torch.from_numpy(qc).cuda()
    dof = torch.from_numpy(qo.view(np.int32)).cuda()
    torch.cuda.synchronize()
    n = ix.query_device(dch.data_ptr(), dof.data_ptr(), len(qo) - 1, distance=2)
    dev = ix.ctx.fetch(n)
    assert np.array_equal(dev.pairs, host.pairs) and np.array_equal(dev.distances, host.distances)
    info = ix.info()
    assert info["n_seqs"] == 100_000 and info["n_records"] > 100_000 and info["max_distance"] == 2
    with xtn.Index(qc, qo, max_distance=1) as small:
        with pytest.raises(xtn.XtnError, match="exceeds the index's maximum distance"):
            small.query(qc, qo, distance=2)


def test_serving_loop_matches_direct_queries(index_setup):
    """Requests arriving over 50 ms, mixed d = 1 / 2 and measures, one larger than the batch
    budget: each request's answer equals a direct query of the same sequences."""
    ix, index_seqs = index_setup
    rng = np.random.default_rng(12)
    reqs = []
    for i in range(24):
        size = int(rng.integers(1, 400)) if i != 7 else 1300
        q = make_queries(index_seqs, size, seed=100 + i)
        c, o = csr(q)
        d = 1 if rng.random() < 0.7 else 2
        m = 1 if i % 5 == 4 else 0
        reqs.append((c, o, d, m, float(rng.uniform(0, 0.05))))
    expected = [ix.query(c, o, distance=d, measure=m) for c, o, d, m, _ in reqs]
    assert sum(len(e.pairs) for e in expected) > 0
    # in real time (arrival times honoured), then with every request ready at once, so that
    # requests of one (distance, measure) share batches and the large one is split
    for realtime in (True, False):
        stats, outs = ix.serve(reqs, max_batch_seqs=1000, realtime=realtime)
        for (c, o, d, m, t), st, out, exp in zip(reqs, stats, outs, expected):
            assert st["status"] == 0
            if realtime:
                assert st["admitted_s"] >= t - 1e-6
            assert st["done_s"] >= st["admitted_s"]
            assert np.array_equal(out.pairs, exp.pairs)
            assert np.array_equal(out.distances, exp.distances)
            assert st["n_out"] == len(exp.pairs)
        if not realtime:
            assert len({st["batch"] for st in stats}) < len(reqs)


@pytest.mark.parametrize("slots", [1, 2, 4])
def test_serving_slots_results_alone_and_in_the_mix(index_setup, slots):
    """Continuous batching: with several slots, batches run at the same time on their own
    streams. Each request's answer equals the same request queried alone, whatever batch and
    slot it joined."""
    ix, index_seqs = index_setup
    rng = np.random.default_rng(31 + slots)
    reqs = []
    for i in range(40):
        size = int(rng.integers(1, 300)) if i % 9 else 3000
        q = make_queries(index_seqs, size, seed=500 + i)
        c, o = csr(q)
        reqs.append((c, o, 1 if rng.random() < 0.7 else 2, 0, float(rng.uniform(0, 0.03))))
    expected = [ix.query(c, o, distance=d, measure=m) for c, o, d, m, _ in reqs]
    for realtime in (True, False):
        stats, outs = ix.serve(reqs, realtime=realtime, slots=slots)
        for st, out, exp in zip(stats, outs, expected):
            assert st["status"] == 0
            assert np.array_equal(out.pairs, exp.pairs) and np.array_equal(out.distances, exp.distances)


def test_small_request_overtakes_a_large_one(index_setup):
    """A large d = 2 batch occupies one slot; small d = 1 requests that arrive while it runs are
    admitted by the other slot and finish before it."""
    ix, index_seqs = index_setup
    big = csr(make_queries(index_seqs, 60_000, seed=1))
    smalls = [csr(make_queries(index_seqs, 20, seed=600 + i)) for i in range(6)]
    reqs = [(big[0], big[1], 2, 0, 0.0)] + [(c, o, 1, 0, 0.001 + 0.0005 * i) for i, (c, o) in enumerate(smalls)]
    ix.serve(reqs, realtime=True, slots=2, keep_results=False)  # warm-up of the slots' buffers
    stats, outs = ix.serve(reqs, realtime=True, slots=2)
    big_done = stats[0]["done_s"]
    assert any(st["done_s"] < big_done for st in stats[1:]), [st["done_s"] for st in stats]
    assert len({st["batch"] for st in stats}) >= 2
    for (c, o, d, m, _), out in zip(reqs, outs):
        exp = ix.query(c, o, distance=d, measure=m)
        assert np.array_equal(out.pairs, exp.pairs) and np.array_equal(out.distances, exp.distances)


def test_serving_on_the_5m_index_equals_offline_runs():
    """The serving configuration's index (5,000,000 generator sequences, d = 2): requests of
    mixed sizes and distances, served with two slots, each equal to the offline search on
    (index sequences followed by the request) restricted to the pairs with one side in each."""
    import torch

    chars, offs = xtn.synth_clusters(20245, 5_300_000, 0.20, 0.02)
    ni = 5_000_000
    ic, io = chars[: offs[ni]], offs[: ni + 1]
    pool_c, pool_o = chars[offs[ni]:], (offs[ni:] - offs[ni]).astype(np.uint32)
    rng = np.random.default_rng(7)
    reqs = []
    for k in range(10):
        size = int(np.exp(rng.uniform(0, np.log(50_000))))
        a = int(rng.integers(0, len(pool_o) - 1 - size))
        o = (pool_o[a : a + size + 1] - pool_o[a]).astype(np.uint32)
        reqs.append((pool_c[pool_o[a] : pool_o[a + size]], o, 1 if k % 3 else 2, 0, 0.002 * k))
    with xtn.Index(ic, io, max_distance=2) as ix:
        stats, outs = ix.serve(reqs, realtime=True, slots=2)
    ctx = xtn.Context(0)
    for (c, o, d, m, _), st, out in zip(reqs, stats, outs):
        assert st["status"] == 0
        uc = np.concatenate([ic, c])
        uo = np.concatenate([io, o[1:] + io[-1]]).astype(np.uint32)
        dch = torch.from_numpy(uc).cuda()
        dof = torch.from_numpy(uo.view(np.int32)).cuda()
        torch.cuda.synchronize()
        m_out = ctx.nn_device(dch.data_ptr(), dof.data_ptr(), len(uo) - 1, d, m)
        r = ctx.fetch(m_out)
        sel = (r.pairs[:, 0] < ni) & (r.pairs[:, 1] >= ni)
        assert np.array_equal(out.pairs, r.pairs[sel])
        assert np.array_equal(out.distances, r.distances[sel])
    ctx.close()
