"""Multi-round searches (the memory model and its rounds).

The reference splits a search into lower-bound rounds sized from free memory
(xtneighbor_streaming/src/xtn.cu:21-26,64-157,383-470). Here a search whose variant records do
not fit the memory budget runs in rounds over contiguous ranges of first-level hash buckets,
with one candidate-pair hash set across the rounds. Forced to many rounds by a small budget or
a small per-round record bound, the output must stay bit-exact against the CPU oracle, with
the dedup of each round overlapped on a second stream or run in turn, with or without the
hash set, and for d = 3 (direct scatter). A budget that cannot hold one first-level bucket is
an error, not a fault.
"""
import numpy as np
import pytest

import oracle as orc
import xtn
from conftest import assert_same_pairs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def clusters60k():
    chars, offs = xtn.synth_clusters(seed=7, n=60_000, cluster_frac=0.2, dup_frac=0.02)
    exp = {m: orc.nn_search(chars, offs, 2, m)[:2] for m in (0, 1)}
    return chars, offs, exp


@pytest.mark.parametrize("overlap", [1, 0])
@pytest.mark.parametrize("measure", [0, 1])
def test_forced_rounds_equal_oracle(clusters60k, overlap, measure):
    chars, offs, exp = clusters60k
    with xtn.Context(0) as ctx:
        one = ctx.perform(chars, offs, distance=2, measure=measure)
        V = ctx.stats()["n_variants"]
        assert ctx.stats()["n_rounds"] == 1
        ctx.set_option("round_overlap", overlap)
        ctx.set_option("max_round_records", V // 10)
        got = ctx.perform(chars, offs, distance=2, measure=measure)
        st = ctx.stats()
    assert st["n_rounds"] >= 8
    assert_same_pairs(got.pairs, got.distances, exp[measure][0], exp[measure][1], f"rounds m={measure}")
    assert_same_pairs(one.pairs, one.distances, exp[measure][0], exp[measure][1], "one round")


def test_memory_budget_forces_rounds(clusters60k):
    chars, offs, exp = clusters60k
    with xtn.Context(0, memory_budget=48 << 20) as ctx:
        got = ctx.perform(chars, offs, distance=2)
        st = ctx.stats()
    assert st["n_rounds"] >= 2
    assert_same_pairs(got.pairs, got.distances, exp[0][0], exp[0][1], "memory budget")


def test_rounds_without_hash_set(clusters60k):
    """pair_dedup = 0: every round's candidates are kept and sorted together."""
    chars, offs, exp = clusters60k
    with xtn.Context(0, pair_dedup=0, max_round_records=700_000) as ctx:
        got = ctx.perform(chars, offs, distance=2)
        assert ctx.stats()["n_rounds"] >= 8
    assert_same_pairs(got.pairs, got.distances, exp[0][0], exp[0][1], "rounds, no hash set")


def test_rounds_table_regrow():
    """pair_dedup = 2 sizes the hash set from the previous search's share of distinct pairs. 400
    copies of one sequence leave a share of about 1 %; the next search, in rounds, has far more
    distinct pairs than that table holds, so an insertion runs out of probes in some round: the
    table grows, is rebuilt from the earlier rounds' distinct pairs, and the round is redone."""
    chars, offs = xtn.synth_clusters(seed=7, n=150_000, cluster_frac=0.2, dup_frac=0.02)
    exp_p, exp_d, _ = orc.nn_search(chars, offs, 2, 0)
    copies_c, copies_o = xtn.pack_sequences(["CASSLGQGAYEQYF"] * 400)
    with xtn.Context(0, pair_dedup=2, max_round_records=1_500_000) as ctx:
        ctx.perform(copies_c, copies_o, distance=2)
        got = ctx.perform(chars, offs, distance=2)
        assert ctx.stats()["n_rounds"] >= 8
    assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, "rounds after regrow")


def test_rounds_d3_direct_scatter():
    chars, offs = xtn.synth_mutants(seed=42, n=10_000, mutant_frac=0.10)
    exp_p, exp_d, _ = orc.nn_search(chars, offs, 3, 0)
    with xtn.Context(0) as ctx:
        ctx.perform(chars, offs, distance=3)
        V = ctx.stats()["n_variants"]
        ctx.set_option("max_round_records", V // 6)
        got = ctx.perform(chars, offs, distance=3)
        assert ctx.stats()["n_rounds"] >= 6
    assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, "rounds d=3")


def test_budget_below_one_bucket_is_an_error(clusters60k):
    chars, offs, _ = clusters60k
    with xtn.Context(0, max_round_records=100) as ctx:
        with pytest.raises(xtn.XtnError, match="cannot hold one first-level bucket") as ei:
            ctx.perform(chars, offs, distance=2)
        assert ei.value.code == xtn.ERR_NOMEM
        ctx.set_option("max_round_records", 0)
        got = ctx.perform(chars, offs, distance=2)
        assert len(got.pairs) > 1000
