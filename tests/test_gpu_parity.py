"""Parity of the CUDA path (through the C ABI) with the CPU oracle and the reference's vectors.

Bit-exact: same (x, y) pairs in the same order and the same int8 distances (NN mode);
same (rep_x, rep_y) entries and uint64 sums (overlap mode).
"""
import numpy as np
import pytest

import oracle as orc
import xtn
from conftest import assert_same_pairs, csr

pytestmark = pytest.mark.gpu


ENGINES = {
    "bucket": {},
    "sort": {"engine": 1},
    # tiny first-level table and shared-memory cap: exercises the bucket split and the
    # sort-based fallback for oversized buckets on small inputs
    "bucket_split_fallback": {"bucket_bits_max": 4, "group_cap": 64, "split_chunk": 2048},
    # buckets loaded into shared memory by plain loads instead of a TMA bulk copy; the larger
    # first-level stage shape; one CTA per split bucket instead of a cluster; classic radix
    # sort passes instead of single-sweep ones; every candidate pair sorted (no hash set)
    "bucket_plain_loads": {"group_tma": 0, "scatter_ctas_per_sm": 1, "stage_chunk": 4096, "split_slices": 1,
                           "onesweep": 0, "pair_dedup": 0},
    # every variant key hashed directly (the d > 2 and no-allocation form) instead of from
    # per-sequence tables; direct first-level scatter
    "bucket_key_hash": {"key_tables": 0},
    # the small grouping shape (buckets of up to 2048 records, 256 threads, six CTAs per SM),
    # the 8192-record first-level stage shape and the verification variant that lists four
    # candidates per lane
    "bucket_small_group": {"group_cap": 2048, "stage_chunk": 8192, "verify_per": 4},
    # the one-pass first-level scatter (generation and partition per chunk) in place of the
    # default two passes (every record generated in sequence order, then partitioned)
    "bucket_one_pass": {"flat_gen": 0},
    # the two-pass split (slice histograms merged in a cluster, exact sub-bucket placement) in
    # place of the default one-pass split into fixed slots of the grouping capacity
    "bucket_two_pass_split": {"split_slotted": 0},
    # the one-pass split on the 8192-record stage (records and ranks kept in registers)
    "bucket_split_8192": {"split_chunk": 8192},
}


@pytest.fixture(scope="module", params=sorted(ENGINES))
def ctx(request):
    c = xtn.Context(0, **ENGINES[request.param])
    yield c
    c.close()


def check_nn(ctx, chars, offs, d, measure, what=""):
    got = ctx.perform(chars, offs, distance=d, measure=measure)
    exp_p, exp_d, _ = orc.nn_search(chars, offs, d, measure)
    assert_same_pairs(got.pairs, got.distances, exp_p, exp_d, what)
    return got


def test_reference_stream4_vectors(ctx, kat):
    """xtneighbor_streaming/test/test_stream4.cu: 7 sequences, two of length 22."""
    k = kat["stream4"]
    chars = np.frombuffer(k["chars"].encode(), np.uint8)
    offs = np.array(k["offsets"], np.uint32)
    got = ctx.perform(chars, offs, distance=k["distance"], measure=k["measure"])
    assert got.pairs.tolist() == k["pairs"]
    assert got.distances.tolist() == k["distances"]


def test_reference_dummy_input(ctx, kat):
    seqs = kat["dummy_input"]["text"].split("\n")[1:-1]
    chars, offs = csr(seqs)
    check_nn(ctx, chars, offs, 1, xtn.LEVENSHTEIN, "dummy")


@pytest.mark.parametrize("d,measure", [(1, 0), (2, 0), (1, 1), (2, 1), (3, 0)])
def test_mutants_10k(ctx, d, measure):
    chars, offs = xtn.synth_mutants(seed=42, n=10_000, mutant_frac=0.10)
    check_nn(ctx, chars, offs, d, measure, f"mutants d={d} m={measure}")


@pytest.mark.parametrize("d,measure", [(2, 0), (2, 1)])
def test_clusters_60k(ctx, d, measure):
    chars, offs = xtn.synth_clusters(seed=7, n=60_000, cluster_frac=0.2, dup_frac=0.02)
    got = check_nn(ctx, chars, offs, d, measure, f"clusters d={d} m={measure}")
    assert len(got.pairs) > 1000


def test_single_and_identical(ctx):
    chars, offs = csr(["CASSLF"])
    got = ctx.perform(chars, offs, distance=1)
    assert len(got.pairs) == 0
    chars, offs = csr(["CASSLF"] * 300 + ["CASSLG"] * 3)
    check_nn(ctx, chars, offs, 1, 0, "identical")


def test_every_sequence_twice(ctx):
    """Each of 40,000 sequences (10% of them mutants of others) appears twice, shuffled, so
    every variant hash is a run of >= 2 records: a first-level bucket or sub-bucket of ~2,500
    records then lists ~1,250 runs, more than the grouping CTA holds, and goes to the
    sort-based regrouping."""
    bc, bo = xtn.synth_mutants(seed=31, n=40_000, mutant_frac=0.10)
    base = [bytes(bc[bo[i] : bo[i + 1]]).decode() for i in range(len(bo) - 1)]
    rng = np.random.default_rng(31)
    seqs = [base[i] for i in rng.permutation(np.repeat(np.arange(len(base)), 2))]
    chars, offs = csr(seqs)
    got = check_nn(ctx, chars, offs, 1, xtn.LEVENSHTEIN, "every sequence twice")
    assert (got.distances == 0).sum() >= 40_000 and (got.distances == 1).sum() > 1000


def test_hash_set_regrows():
    """Large candidate hash sets are sized from the previous search's share of distinct pairs
    (pair_dedup=2 applies that sizing at any size). A search where every pair repeats ~100
    times (400 copies of one sequence, d=2) leaves a share of about 1 %; the next search, with
    far more distinct pairs than that table holds, must redo the pass with a larger one."""
    ctx = xtn.Context(0, pair_dedup=2)
    chars, offs = csr(["CASSLGQGAYEQYF"] * 400)
    check_nn(ctx, chars, offs, 2, 0, "400 copies")
    # ~180k distinct pairs: more than the 2^16-slot table the copies' share asks for
    chars, offs = xtn.synth_clusters(seed=7, n=150_000, cluster_frac=0.2, dup_frac=0.02)
    got = check_nn(ctx, chars, offs, 2, 0, "after the copies")
    assert len(got.pairs) > 40_000
    ctx.close()


def test_invalid_offsets_rejected(ctx):
    """A sequence of 0 or more than 500 residues is rejected with its index, and the context
    stays usable."""
    chars, offs = csr(["CASSLF", "CASS", "CASSLG"])
    bad = offs.copy()
    bad[2] = bad[1]  # sequence 1 empty
    with pytest.raises(xtn.XtnError, match="sequence 1 has an invalid length"):
        ctx.perform(chars, bad, distance=1)
    lc, lo = csr(["CASSLF", "A" * 501])
    with pytest.raises(xtn.XtnError, match="sequence 1 has an invalid length"):
        ctx.perform(lc, lo, distance=1)
    check_nn(ctx, chars, offs, 1, 0, "after rejected inputs")


def test_short_sequences_large_d(ctx):
    """d >= L: the empty variant is shared by every short sequence."""
    rng = np.random.default_rng(1)
    seqs = ["".join(rng.choice(list("ACDE"), int(rng.integers(1, 5)))) for _ in range(400)]
    chars, offs = csr(seqs)
    for d in (1, 2, 3, 4, 6):
        for m in (0, 1):
            check_nn(ctx, chars, offs, d, m, f"short d={d} m={m}")


def test_runs_and_long_sequences(ctx):
    rng = np.random.default_rng(2)
    seqs = []
    for _ in range(600):
        L = int(rng.integers(15, 90))
        s = "".join(rng.choice(list("AAAAC"), L))
        seqs.append(s)
    for i in range(0, 600, 3):  # near copies beyond the 18-residue key and beyond 64
        s = list(seqs[i])
        s[int(rng.integers(0, len(s)))] = "D"
        seqs.append("".join(s))
    chars, offs = csr(seqs)
    for d in (1, 2, 3):
        for m in (0, 1):
            check_nn(ctx, chars, offs, d, m, f"long d={d} m={m}")


def test_hamming_signed_char_wrap(ctx):
    """Equal-length sequences >= 128 residues whose mismatch count wraps the reference's
    signed char: reported only when the 18-residue prefixes share a variant."""
    base = "C" * 18
    a = base + "A" * 182
    b = base + "D" * 182  # 182 mismatches -> (int8)182 = -74 <= d: reported (shared prefix)
    c = "E" * 18 + "A" * 182
    e = "E" * 18 + "D" * 182  # same, prefix shared with c
    f = "G" * 200  # 200 mismatches vs a, but no shared prefix variant: not a candidate
    chars, offs = csr([a, b, c, e, f])
    got = check_nn(ctx, chars, offs, 2, 1, "wrap")
    assert [0, 1] in got.pairs.tolist()


def test_overlap_reference_vectors(ctx, kat):
    k = kat["overlap_init"]
    chars = np.frombuffer(k["chars"].encode(), np.uint8)
    offs = np.array(k["offsets"], np.uint32)
    got = ctx.perform(chars, offs, distance=1, info=np.array(k["info"], np.int32), n_reps=2)
    exp_p, exp_s = orc.overlap_search(chars, offs, k["info"], 1, 0)
    assert got.pairs.tolist() == exp_p.tolist()
    assert got.frequencies.tolist() == exp_s.tolist()


@pytest.mark.parametrize("d,measure", [(1, 0), (1, 1), (2, 0)])
def test_overlap_synthetic(ctx, d, measure):
    chars, offs, info, reps = xtn.synth_repertoires(seed=5, n_reps=12, min_size=200, max_size=4000, shared=0.2)
    got = ctx.perform(chars, offs, distance=d, measure=measure, info=info, n_reps=len(reps))
    exp_p, exp_s = orc.overlap_search(chars, offs, info, d, measure)
    assert got.pairs.tolist() == exp_p.tolist()
    assert np.array_equal(got.frequencies, exp_s)


def test_overlap_negative_counts_wrap(ctx):
    """Counts may be negative (strtol accepts them); products and sums wrap like size_t."""
    seqs = ["CAAA", "CADA", "CAAA", "CDKD", "CAAK"]
    chars, offs = csr(seqs)
    info = np.array([[-3, 0, 0], [4, 0, 1], [2**31 - 1, 1, 2], [-6, 1, 3], [7, 1, 4]], np.int32)
    got = ctx.perform(chars, offs, distance=1, info=info, n_reps=2)
    exp_p, exp_s = orc.overlap_search(chars, offs, info, 1, 0)
    assert got.pairs.tolist() == exp_p.tolist()
    assert np.array_equal(got.frequencies, exp_s)


def test_context_reuse_and_device_entry(ctx):
    import torch

    chars, offs = xtn.synth_clusters(seed=99, n=20_000)
    a = ctx.perform(chars, offs, distance=2)
    small_c, small_o = xtn.synth_mutants(seed=3, n=500)
    ctx.perform(small_c, small_o, distance=1)
    dch = torch.from_numpy(chars).cuda()
    dof = torch.from_numpy(offs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    n = ctx.nn_device(dch.data_ptr(), dof.data_ptr(), len(offs) - 1, distance=2)
    b = ctx.fetch(n)
    assert_same_pairs(b.pairs, b.distances, a.pairs, a.distances, "device entry")
    st = ctx.stats()
    assert st["n_out"] == len(a.pairs) and st["n_variants"] > 0


def test_overlap_device_entry(ctx):
    """xtn_context_overlap_device (inputs in device memory) equals the host-buffer entry; a
    repertoire id outside [0, R) is reported with the first offending row."""
    import torch

    chars, offs, info, reps = xtn.synth_repertoires(seed=11, n_reps=6, min_size=300, max_size=3000, shared=0.2)
    a = ctx.perform(chars, offs, distance=1, info=info, n_reps=len(reps))
    dch = torch.from_numpy(chars).cuda()
    dof = torch.from_numpy(offs.view(np.int32)).cuda()
    dinf = torch.from_numpy(np.ascontiguousarray(info)).cuda()
    torch.cuda.synchronize()
    m = ctx.overlap_device(dch.data_ptr(), dof.data_ptr(), len(offs) - 1, dinf.data_ptr(), len(reps), distance=1)
    b = ctx.fetch_overlap(m)
    assert a.pairs.tolist() == b.pairs.tolist()
    assert np.array_equal(a.frequencies, b.frequencies)
    bad = info.copy()
    bad[9, 1] = -1
    bad[7, 1] = len(reps)
    with pytest.raises(xtn.XtnError, match="out of range at row 7$"):
        ctx.perform(chars, offs, distance=1, info=bad, n_reps=len(reps))


def test_autotune_keeps_results_exact():
    """The autotuner picks a bucket-engine shape by timing; the search stays bit-exact."""
    import torch

    chars, offs = xtn.synth_clusters(seed=13, n=50_000)
    ctx = xtn.Context(0)
    dch = torch.from_numpy(chars).cuda()
    dof = torch.from_numpy(offs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    report = ctx.autotune(dch.data_ptr(), dof.data_ptr(), len(offs) - 1, distance=2, repeats=1)
    assert "stage_chunk=" in report and "best of" in report
    check_nn(ctx, chars, offs, 2, 0, "after autotune")
    ctx.close()
