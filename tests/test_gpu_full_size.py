"""Parity at the benchmark's full sizes.

1,000,000 sequences, Levenshtein d = 2 (the benchmark workload): bit-exact against the CPU
oracle, every pair and every distance.

10,000,000 sequences, d = 2, Levenshtein and Hamming (too large for a full oracle run here):
properties that hold at any size.
  - The hash-bucket engine and the full-sort engine return identical results.
  - Pairs are strictly increasing in (x, y), with x < y.
  - The oracle recomputes the distances of a random sample of pairs.
  - Every Hamming pair is also a Levenshtein pair, at a Levenshtein distance no larger.
  - For sampled query sequences, the exhaustive neighbour scan (oracle.brute_neighbors)
    finds exactly the reported pairs that involve them. This is completeness and soundness
    for those queries.
  - Forced into eight rounds, the search returns exactly the one-round result (which the
    reference binary matches byte for byte, tests/test_gpu_reference_full_size.py).

10,000,000 sequences at d = 3 (about 5.8e9 deletion variants, more than one round can hold in
32-bit positions): the search runs in rounds and its result has the same properties.
"""
import numpy as np
import pytest

import oracle as orc
import xtn
from conftest import assert_same_pairs

pytestmark = pytest.mark.gpu


def check_sorted_unique(pairs):
    assert (pairs[:, 0] < pairs[:, 1]).all()
    key = pairs[:, 0].astype(np.int64) << 32 | pairs[:, 1].astype(np.int64)
    assert (np.diff(key) > 0).all()


def check_sample_distances(chars, offs, pairs, dist, measure, k=2000, seed=0):
    rng = np.random.default_rng(seed)
    fn = orc.hamming if measure else orc.levenshtein
    for i in rng.choice(len(pairs), size=min(k, len(pairs)), replace=False):
        x, y = pairs[i]
        a = bytes(chars[offs[x] : offs[x + 1]]).decode()
        b = bytes(chars[offs[y] : offs[y + 1]]).decode()
        assert fn(a, b) == dist[i], (x, y)


def check_queries(chars, offs, pairs, dist, d, measure, n_random=24, seed=1):
    rng = np.random.default_rng(seed)
    n = len(offs) - 1
    q = np.unique(np.concatenate([rng.choice(n, n_random, replace=False),
                                  pairs[rng.choice(len(pairs), 8, replace=False), 0]]).astype(np.int32))
    exp = orc.brute_neighbors(chars, offs, q, d, measure)
    sel = np.isin(pairs[:, 0], q) | np.isin(pairs[:, 1], q)
    got = np.concatenate([pairs[sel], dist[sel, None].astype(np.int32)], axis=1)
    assert np.array_equal(got, exp)
    assert len(exp) > 0


def test_1m_leven_d2_equals_oracle():
    chars, offs = xtn.synth_clusters(20241, 1_000_000, 0.20, 0.02)
    ctx = xtn.Context(0)
    got = ctx.perform(chars, offs, distance=2)
    ctx.close()
    exp_p, exp_d, _ = orc.nn_search(chars, offs, 2, 0)
    assert len(exp_p) > 100_000
    assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, "1M leven d=2")


@pytest.fixture(scope="module")
def ten_million():
    return xtn.synth_clusters(20242, 10_000_000, 0.20, 0.02)


@pytest.fixture(scope="module")
def ten_million_results(ten_million):
    chars, offs = ten_million
    ctx = xtn.Context(0)
    out = {m: ctx.perform(chars, offs, distance=2, measure=m) for m in (xtn.LEVENSHTEIN, xtn.HAMMING)}
    ctx.close()
    return out


@pytest.mark.parametrize("measure", [xtn.LEVENSHTEIN, xtn.HAMMING])
def test_10m_d2_properties(ten_million, ten_million_results, measure):
    chars, offs = ten_million
    r = ten_million_results[measure]
    assert len(r.pairs) > 500_000
    check_sorted_unique(r.pairs)
    assert (r.distances >= 0).all() and (r.distances <= 2).all()
    check_sample_distances(chars, offs, r.pairs, r.distances, measure)
    check_queries(chars, offs, r.pairs, r.distances, 2, measure)


def test_10m_engines_agree(ten_million, ten_million_results):
    chars, offs = ten_million
    ctx = xtn.Context(0, engine=1)
    s = ctx.perform(chars, offs, distance=2)
    ctx.close()
    b = ten_million_results[xtn.LEVENSHTEIN]
    assert_same_pairs(s.pairs, s.distances, b.pairs, b.distances, "10M sort vs bucket engine")


def test_10m_hamming_within_levenshtein(ten_million_results):
    lev, ham = ten_million_results[xtn.LEVENSHTEIN], ten_million_results[xtn.HAMMING]
    lk = lev.pairs[:, 0].astype(np.int64) << 32 | lev.pairs[:, 1].astype(np.int64)
    hk = ham.pairs[:, 0].astype(np.int64) << 32 | ham.pairs[:, 1].astype(np.int64)
    pos = np.searchsorted(lk, hk)
    assert (pos < len(lk)).all() and (lk[pos] == hk).all()
    assert (lev.distances[pos] <= ham.distances).all()


def test_10m_rounds_equal_one_round(ten_million, ten_million_results):
    chars, offs = ten_million
    b = ten_million_results[xtn.LEVENSHTEIN]
    ctx = xtn.Context(0)
    ctx.set_option("max_round_records", 1_096_096_457 // 8 + 1)
    r = ctx.perform(chars, offs, distance=2)
    assert ctx.stats()["n_rounds"] >= 8
    ctx.close()
    assert_same_pairs(r.pairs, r.distances, b.pairs, b.distances, "10M, eight rounds vs one")


def test_10m_d3_completes_in_rounds(ten_million):
    chars, offs = ten_million
    ctx = xtn.Context(0)
    r = ctx.perform(chars, offs, distance=3)
    st = ctx.stats()
    ctx.close()
    assert st["n_variants"] > 2**32 and st["n_rounds"] >= 2
    assert len(r.pairs) > len(chars) // 100
    check_sorted_unique(r.pairs)
    assert (r.distances >= 0).all() and (r.distances <= 3).all()
    check_sample_distances(chars, offs, r.pairs, r.distances, 0, k=1000)
    check_queries(chars, offs, r.pairs, r.distances, 3, 0, n_random=8)
