"""The batched/persistent form (context option "graph"): the whole search captured into one
CUDA graph whose kernels read every data-dependent size on the device, replayed per search.
It must return exactly what the plain form returns (which the parity suite pins to the oracle
and the reference), on first use (plain search, then capture), on every replay, after the
input changes in place (a replay that outgrows its capacities is redone by the plain form),
and it must reject invalid lengths like the plain form.
"""
import numpy as np
import pytest

import oracle as orc
import xtn
from conftest import assert_same_pairs

pytestmark = pytest.mark.gpu


def on_device(torch, chars, offs, pad=0):
    dch = torch.zeros(len(chars) + 64 + pad, dtype=torch.uint8, device="cuda")
    dch[: len(chars)] = torch.from_numpy(chars).cuda()
    dof = torch.from_numpy(offs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    return dch, dof


@pytest.mark.parametrize("kind,n,d,measure", [("clusters", 60_000, 2, 0), ("clusters", 60_000, 2, 1),
                                              ("mutants", 10_000, 1, 0), ("mutants", 10_000, 3, 0)])
def test_graph_form_equals_oracle_on_every_replay(kind, n, d, measure):
    import torch

    chars, offs = (xtn.synth_clusters(seed=7, n=n) if kind == "clusters" else xtn.synth_mutants(seed=42, n=n))
    exp_p, exp_d, _ = orc.nn_search(chars, offs, d, measure)
    dch, dof = on_device(torch, chars, offs)
    with xtn.Context(0, graph=1) as ctx:
        for rep in range(4):  # plain + capture, then three replays
            m = ctx.nn_device(dch.data_ptr(), dof.data_ptr(), n, d, measure)
            got = ctx.fetch(m)
            assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, f"graph form, search {rep}")
        st = ctx.stats()
        assert st["n_launches"] > 10 and st["n_out"] == len(exp_p)


def test_graph_form_redoes_a_replay_that_outgrows_its_capacities():
    """Same device buffers, new contents: a replay whose variants or candidates exceed the
    captured capacities is redone by the plain form (and the graph re-sized)."""
    import torch

    small_c, small_o = xtn.synth_mutants(seed=5, n=20_000, mutant_frac=0.01)
    big_c, big_o = xtn.synth_clusters(seed=6, n=20_000, cluster_frac=0.9, dup_frac=0.2)
    dch, dof = on_device(torch, small_c, small_o, pad=max(0, len(big_c) - len(small_c)))
    with xtn.Context(0, graph=1) as ctx:
        for c_, o_ in ((small_c, small_o), (big_c, big_o), (big_c, big_o), (small_c, small_o)):
            dch[: len(c_)] = torch.from_numpy(c_).cuda()
            dof.copy_(torch.from_numpy(o_.view(np.int32)).cuda())
            torch.cuda.synchronize()
            exp_p, exp_d, _ = orc.nn_search(c_, o_, 2, 0)
            m = ctx.nn_device(dch.data_ptr(), dof.data_ptr(), len(o_) - 1, 2, 0)
            got = ctx.fetch(m)
            assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, "graph form after new contents")


def test_graph_form_rejects_bad_lengths():
    import torch

    chars, offs = xtn.synth_mutants(seed=9, n=5000)
    dch, dof = on_device(torch, chars, offs)
    with xtn.Context(0, graph=1) as ctx:
        ctx.nn_device(dch.data_ptr(), dof.data_ptr(), 5000, 2, 0)  # plain + capture
        bad = offs.copy()
        bad[1001] = bad[1000]  # sequence 1000 empty
        dof.copy_(torch.from_numpy(bad.view(np.int32)).cuda())
        torch.cuda.synchronize()
        with pytest.raises(xtn.XtnError, match="sequence 1000 has an invalid length"):
            ctx.nn_device(dch.data_ptr(), dof.data_ptr(), 5000, 2, 0)
        dof.copy_(torch.from_numpy(offs.view(np.int32)).cuda())
        torch.cuda.synchronize()
        m = ctx.nn_device(dch.data_ptr(), dof.data_ptr(), 5000, 2, 0)
        exp_p, exp_d, _ = orc.nn_search(chars, offs, 2, 0)
        got = ctx.fetch(m)
        assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, "graph form after a rejected input")


@pytest.mark.parametrize("per", [1, 8])
def test_verification_variants_exact(per):
    chars, offs = xtn.synth_clusters(seed=7, n=60_000)
    exp_p, exp_d, _ = orc.nn_search(chars, offs, 2, 0)
    with xtn.Context(0, verify_per=per) as ctx:
        got = ctx.perform(chars, offs, distance=2)
    assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, f"verify_per={per}")


def test_autotune_cache_by_input_class():
    """Option autotune: the first search of an input class runs the autotuner (which may pick
    the graph form), later searches of the class reuse its choice; results stay exact."""
    import torch

    chars, offs = xtn.synth_clusters(seed=13, n=50_000)
    exp_p, exp_d, _ = orc.nn_search(chars, offs, 2, 0)
    dch, dof = on_device(torch, chars, offs)
    with xtn.Context(0, autotune=1) as ctx:
        for _ in range(3):
            m = ctx.nn_device(dch.data_ptr(), dof.data_ptr(), 50_000, 2, 0)
            got = ctx.fetch(m)
            assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, "autotuned")
    with xtn.Context(0) as ctx:
        report = ctx.autotune(dch.data_ptr(), dof.data_ptr(), 50_000, distance=2, repeats=1)
        assert "verify_per=" in report and "graph=" in report and "median_len=" in report


def _overlap_on_device(torch, chars, offs, info, pad=0):
    dch, dof = on_device(torch, chars, offs, pad)
    dinf = torch.from_numpy(np.ascontiguousarray(info)).cuda()
    torch.cuda.synchronize()
    return dch, dof, dinf


@pytest.mark.parametrize("d,measure", [(1, 0), (2, 0), (1, 1)])
def test_overlap_graph_form_equals_oracle_on_every_replay(d, measure):
    """Overlap mode in the graph form (string merge, diagonal term, the search over the unique
    strings, cross term and matrix in one captured sequence): the plain run plus capture, then
    replays, all equal to the oracle."""
    import torch

    chars, offs, info, reps = xtn.synth_repertoires(seed=21, n_reps=16, min_size=500, max_size=8000, shared=0.2)
    exp_p, exp_s = orc.overlap_search(chars, offs, info, d, measure)
    dch, dof, dinf = _overlap_on_device(torch, chars, offs, info)
    n = len(offs) - 1
    with xtn.Context(0, graph=1) as ctx:
        for rep in range(4):
            m = ctx.overlap_device(dch.data_ptr(), dof.data_ptr(), n, dinf.data_ptr(), len(reps), d, measure)
            got = ctx.fetch_overlap(m)
            assert got.pairs.tolist() == exp_p.tolist(), f"graph form, run {rep}"
            assert np.array_equal(got.frequencies, exp_s), f"graph form, run {rep}"
        st = ctx.stats()
        assert st["n_launches"] > 20 and st["n_out"] == len(exp_p)


def test_overlap_graph_form_redoes_changed_contents():
    """Same device buffers, new contents: a replay whose unique-string count or search sizes
    differ from the capture is redone by the plain form; frequencies changed in place are picked
    up by the replay itself."""
    import torch

    a = xtn.synth_repertoires(seed=31, n_reps=8, min_size=400, max_size=5000, shared=0.2)
    b = xtn.synth_repertoires(seed=32, n_reps=8, min_size=400, max_size=5000, shared=0.3)
    n = min(len(a[1]), len(b[1])) - 1
    cases = []
    for chars, offs, info, reps in (a, b):
        offs = offs[: n + 1].copy()
        chars = chars[: offs[-1]].copy()
        cases.append((chars, offs, info[:n].copy(), len(reps)))
    pad = max(len(c[0]) for c in cases)
    dch, dof, dinf = _overlap_on_device(torch, cases[0][0], cases[0][1], cases[0][2], pad=pad)
    R = max(c[3] for c in cases)
    with xtn.Context(0, graph=1) as ctx:
        order = (0, 0, 1, 1, 0)
        for k, which in enumerate(order):
            chars, offs, info, _ = cases[which]
            if k == 1:  # the same strings with other frequencies
                info = info.copy()
                info[:, 0] = (info[:, 0] * 3 + 1).astype(np.int32)
            dch[: len(chars)] = torch.from_numpy(chars).cuda()
            dof.copy_(torch.from_numpy(offs.view(np.int32)).cuda())
            dinf.copy_(torch.from_numpy(np.ascontiguousarray(info)).cuda())
            torch.cuda.synchronize()
            exp_p, exp_s = orc.overlap_search(chars, offs, info, 1, 0)
            m = ctx.overlap_device(dch.data_ptr(), dof.data_ptr(), n, dinf.data_ptr(), R, 1, 0)
            got = ctx.fetch_overlap(m)
            assert got.pairs.tolist() == exp_p.tolist(), f"run {k}"
            assert np.array_equal(got.frequencies, exp_s), f"run {k}"


def test_overlap_graph_form_rejects_bad_input_like_the_plain_form():
    import torch

    chars, offs, info, reps = xtn.synth_repertoires(seed=41, n_reps=6, min_size=300, max_size=3000, shared=0.2)
    n = len(offs) - 1
    dch, dof, dinf = _overlap_on_device(torch, chars, offs, info)
    exp_p, exp_s = orc.overlap_search(chars, offs, info, 1, 0)
    with xtn.Context(0, graph=1) as ctx:
        ctx.overlap_device(dch.data_ptr(), dof.data_ptr(), n, dinf.data_ptr(), len(reps), 1, 0)  # plain + capture
        bad = info.copy()
        bad[9, 1] = -1
        bad[7, 1] = len(reps)
        dinf.copy_(torch.from_numpy(bad).cuda())
        torch.cuda.synchronize()
        with pytest.raises(xtn.XtnError, match="out of range at row 7$"):
            ctx.overlap_device(dch.data_ptr(), dof.data_ptr(), n, dinf.data_ptr(), len(reps), 1, 0)
        dinf.copy_(torch.from_numpy(info).cuda())
        badoffs = offs.copy()
        badoffs[501] = badoffs[500]  # sequence 500 empty
        dof.copy_(torch.from_numpy(badoffs.view(np.int32)).cuda())
        torch.cuda.synchronize()
        with pytest.raises(xtn.XtnError, match="sequence 500 has an invalid length"):
            ctx.overlap_device(dch.data_ptr(), dof.data_ptr(), n, dinf.data_ptr(), len(reps), 1, 0)
        dof.copy_(torch.from_numpy(offs.view(np.int32)).cuda())
        torch.cuda.synchronize()
        m = ctx.overlap_device(dch.data_ptr(), dof.data_ptr(), n, dinf.data_ptr(), len(reps), 1, 0)
        got = ctx.fetch_overlap(m)
        assert got.pairs.tolist() == exp_p.tolist()
        assert np.array_equal(got.frequencies, exp_s)


def test_graph_is_recaptured_after_buffers_grow():
    """A search through another entry point (here a larger host-buffer search) may reallocate
    the context's buffers; the next device search must not replay a graph that holds the old
    addresses."""
    import torch

    chars, offs = xtn.synth_mutants(seed=51, n=8000)
    big_c, big_o = xtn.synth_clusters(seed=52, n=120_000)
    dch, dof = on_device(torch, chars, offs)
    exp_p, exp_d, _ = orc.nn_search(chars, offs, 2, 0)
    with xtn.Context(0, graph=1) as ctx:
        for _ in range(2):
            got = ctx.fetch(ctx.nn_device(dch.data_ptr(), dof.data_ptr(), 8000, 2, 0))
            assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, "before")
        ctx.perform(big_c, big_o, distance=2)
        for k in range(2):
            got = ctx.fetch(ctx.nn_device(dch.data_ptr(), dof.data_ptr(), 8000, 2, 0))
            assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, f"after the larger search, run {k}")
