"""The CPU oracle against the reference's own unit-test vectors (xtneighbor_streaming/test/*.cu).

These pin the oracle before it is trusted as the checker of the CUDA path.
"""
import numpy as np
import pytest

import oracle as orc
from conftest import csr


def test_char_encode(kat):
    for c, v in kat["char_encode"]["cases"]:
        assert orc.char_encode(c) == v


def test_str_encode_decode_len(kat):
    assert list(orc.str_encode("A")) == kat["str_encode"]["A"]
    s = kat["str_encode"]["roundtrip"]
    assert orc.str_decode(orc.str_encode(s)) == s
    assert orc.len_decode(orc.str_encode("ACC")) == kat["len_decode"]["ACC"]


def test_remove_char(kat):
    k = kat["remove_char"]
    w = orc.str_encode(k["input"])
    for p, exp in enumerate(k["expected"]):
        assert orc.str_decode(orc.remove_char(w, p)) == exp
    w2 = orc.str_encode(k["input2"])
    for p, exp in enumerate(k["expected2"]):
        assert orc.str_decode(orc.remove_char(w2, p)) == exp


def test_generate_combination_order(kat):
    for case in kat["generate_combination"]["cases"]:
        assert orc.expand_keys(case["input"], case["distance"]) == case["expected"]


def test_stream1(kat):
    k = kat["stream1"]
    keys, ids, hist = orc.stream1(k["seqs"], k["distance"], nbins=16)
    assert keys == k["keys"]
    assert list(ids) == k["ids"]
    assert hist.sum() == len(k["keys"])


def test_stream2(kat):
    k = kat["stream2"]
    keys, ids, hist, rows = orc.stream2(k["keys_in"], k["ids_in"], k["seq_len"], 16, k["max_row"])
    assert keys == k["keys_out"]
    assert list(ids) == k["ids_out"]
    assert list(hist) == k["histogram"]
    assert list(rows) == k["row_split"]


def test_stream3(kat):
    k = kat["stream3"]
    pairs, hist, keys_left, ids_left = orc.stream3(k["keys_in"], k["ids_in"], k["lowerbound"], k["seq_len"], 16)
    assert pairs.tolist() == k["pairs"]
    assert list(hist) == k["histogram"]
    assert keys_left == k["keys_left"]
    assert list(ids_left) == k["ids_left"]


def test_stream4(kat):
    k = kat["stream4"]
    chars = np.frombuffer(k["chars"].encode(), np.uint8)
    offs = np.array(k["offsets"], np.uint32)
    n = len(offs) - 1
    allpairs = [(i, j) for i in range(n) for j in range(i + 1, n)]
    pairs, dist = orc.stream4_nn(chars, offs, n, allpairs, k["distance"], k["measure"])
    assert pairs.tolist() == k["pairs"]
    assert list(dist) == k["distances"]


def test_stream4_whole_search(kat):
    """The same 7 sequences through the whole-search composition."""
    k = kat["stream4"]
    chars = np.frombuffer(k["chars"].encode(), np.uint8)
    offs = np.array(k["offsets"], np.uint32)
    pairs, dist, _ = orc.nn_search(chars, offs, k["distance"], k["measure"])
    assert pairs.tolist() == k["pairs"]
    assert list(dist) == k["distances"]


def test_overlap_init(kat):
    k = kat["overlap_init"]
    chars = np.frombuffer(k["chars"].encode(), np.uint8)
    offs = np.array(k["offsets"], np.uint32)
    u, info_sorted, cum, keys, entries, sums = orc.overlap_init(chars, offs, k["info"])
    assert u == k["unique"]
    assert info_sorted.tolist() == k["info_sorted"]
    assert list(cum) == k["cum_counts"]
    assert [orc.str_decode(w) for w in keys] == k["unique_seqs"]
    assert entries.tolist() == k["entries"]
    assert [int(x) for x in sums] == k["sums"]


def test_deduplicate_full_length(kat):
    k = kat["deduplicate_full_length"]
    chars = np.frombuffer(k["chars"].encode(), np.uint8)
    offs = np.array(k["offsets"], np.uint32)
    u, info_sorted, cum, keys, _, _ = orc.overlap_init(chars, offs, k["info"])
    assert u == k["unique"]
    counts = np.diff(np.concatenate([[0], cum]))
    assert list(counts) == k["counts"]
    assert [orc.str_decode(w) for w in keys] == k["unique_seqs"]
    assert info_sorted.tolist() == k["info_sorted"]


def test_stream4_overlap(kat):
    k = kat["stream4_overlap"]
    chars = np.frombuffer(k["chars"].encode(), np.uint8)
    offs = np.array(k["offsets"], np.uint32)
    n = len(k["cum_counts"])
    allpairs = [(i, j) for i in range(n) for j in range(i + 1, n)]
    entries, sums = orc.stream4_overlap(chars, offs, k["info_sorted"], k["cum_counts"], allpairs, k["distance"], k["measure"])
    assert entries.tolist() == k["entries"]
    assert [int(x) for x in sums] == k["sums"]


def test_overlap_whole_search_matches_stages(kat):
    """Whole overlap search = diagonal (overlap_init) + cross term (stream4_overlap)."""
    k = kat["overlap_init"]
    chars = np.frombuffer(k["chars"].encode(), np.uint8)
    offs = np.array(k["offsets"], np.uint32)
    entries, sums = orc.overlap_search(chars, offs, k["info"], 1, 0)
    # CAAA(r0,f3) CADA(r0,f4) CAAA(r1,f5) CDKD(r1,f6); CAAA~CADA at distance 1:
    # diagonal {(0,0):25,(0,1):15,(1,1):61}; cross CAAA x CADA: (3*4*2 -> (0,0)), (5*4 -> (0,1))
    assert entries.tolist() == [[0, 0], [0, 1], [1, 1]]
    assert [int(x) for x in sums] == [25 + 24, 15 + 20, 61]


def test_bin_packing(kat):
    for case in kat["bin_packing_offsets"]["cases"]:
        per, out = orc.bin_packing_offsets(np.array(case["hist"]), case["exponent"])
        assert per == len(case["expected"][0])
        assert out.tolist() == case["expected"]
    k = kat["bin_packing_lowerbounds"]
    assert orc.bin_packing_lowerbounds(np.array(k["hist"]), k["seq_len"], k["exponent"]).tolist() == k["expected"]


def test_histogram_exact(kat):
    k = kat["histogram"]
    a = k["no_loss"]
    v = np.arange(a["n"], dtype=np.int64) % a["seq_len"]
    assert orc.histogram(v, a["bins"], 0, a["seq_len"]).sum() == a["n"]
    b = k["large_index"]
    v = b["seq_len"] - 1 - (np.arange(b["n"], dtype=np.int64) % b["seq_len"])
    assert orc.histogram(v, b["bins"], 0, b["seq_len"]).sum() == b["n"]
    c = k["vs_edges"]
    v = (np.arange(c["n"], dtype=np.int64) * c["stride"]) % c["seq_len"]
    # bin i holds [ceil(i*range/bins), ceil((i+1)*range/bins)) (test_bin_packing.cu:126-166)
    edges = (np.arange(c["bins"], dtype=np.int64) * c["seq_len"] + c["bins"] - 1) // c["bins"]
    expected = np.bincount(np.searchsorted(edges, v, side="right") - 1, minlength=c["bins"])
    assert np.array_equal(orc.histogram(v, c["bins"], 0, c["seq_len"]), expected)


def test_distances_reference_semantics():
    assert orc.levenshtein("CAAA", "CADA") == 1
    assert orc.levenshtein("CASSLGF", "CASSLF") == 1
    assert orc.hamming("CAAA", "CAA") == 77
    assert orc.hamming("CAAA", "CADA") == 1
    # the reference's signed-char mismatch counter wraps past 127
    a, b = "A" * 200, "C" * 200
    assert orc.hamming(a, b) == np.int8(np.uint8(200))


def test_whole_search_equals_bruteforce_small():
    """orc_nn_search on random short sequences = exhaustive search (completeness of the keys)."""
    rng = np.random.default_rng(7)
    alphabet = np.array(list("ACDEFGHIKLMNPQRSTVWY"))
    seqs = []
    for _ in range(300):
        L = int(rng.integers(3, 24))
        base = "".join(rng.choice(alphabet[:5], L))
        seqs.append(base)
    chars, offs = csr(seqs)
    for d in (1, 2):
        pairs, dist, _ = orc.nn_search(chars, offs, d, 0)
        exp = [(i, j, orc.levenshtein(seqs[i], seqs[j])) for i in range(len(seqs)) for j in range(i + 1, len(seqs))]
        exp = [(i, j, v) for i, j, v in exp if v <= d]
        assert pairs.tolist() == [[i, j] for i, j, _ in exp]
        assert dist.tolist() == [v for _, _, v in exp]
