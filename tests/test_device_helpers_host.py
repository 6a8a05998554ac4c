"""The product's shared host/device helpers (xt-neighbor_b200/csrc/xtn_common.cuh), compiled
for the CPU into tests/hostcheck/libhostcheck.so, against the oracle and brute force.

Covers: run-prefix variant enumeration gives exactly the set of distinct strings of the
reference's variant multiset; the closed-form variant count; Myers' bit-vector Levenshtein
and the banded-exit DP; the reference's Hamming (77 sentinel, signed-char wrap); and the
prefix-shares-a-variant predicate.
"""
import ctypes
import itertools
import os

import numpy as np
import pytest

import oracle as orc

HC = os.path.join(os.path.dirname(__file__), "hostcheck", "libhostcheck.so")
pytestmark = pytest.mark.skipif(not os.path.exists(HC), reason="hostcheck helper not built")


@pytest.fixture(scope="module")
def hc():
    lib = ctypes.CDLL(HC)
    lib.hc_variants.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    lib.hc_tri_row_start.restype = ctypes.c_uint64
    lib.hc_tri_row_start.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
    lib.hc_key_hash.restype = ctypes.c_uint64
    return lib


def variants(hc, s, d):
    n = hc.hc_variants(s.encode(), len(s), d, None, None, 0)
    buf = ctypes.create_string_buffer(19 * n)
    hs = np.zeros(n, np.uint64)
    hc.hc_variants(s.encode(), len(s), d, buf, hs.ctypes.data_as(ctypes.c_void_p), n)
    raw = buf.raw
    out = [raw[19 * i : 19 * i + 19].split(b"\0")[0].decode() for i in range(n)]
    return out, hs


def rand_seqs(rng, n, lo=1, hi=26, alpha="ACDEFGHIKLMNPQRSTVWY"):
    out = []
    for _ in range(n):
        L = int(rng.integers(lo, hi))
        sub = alpha[: int(rng.integers(2, len(alpha) + 1))]
        out.append("".join(rng.choice(list(sub), L)))
    return out


def test_variant_set_equals_reference_multiset(hc):
    rng = np.random.default_rng(3)
    for s in rand_seqs(rng, 500):
        for d in (1, 2, 3, 4):
            got, hashes = variants(hc, s, d)
            ref = orc.expand_keys(s, d)
            assert set(got) == set(ref), (s, d)
            assert hc.hc_variant_count(s.encode(), len(s), d) == len(got), (s, d)
            # equal strings hash equally
            hm = {}
            for g, h in zip(got, hashes):
                assert hm.setdefault(g, int(h)) == int(h)


def test_flat_variant_index_matches_enumeration(hc):
    """variant_at(v), v = 0..count-1 (the staged scatter's parallel decode) yields exactly the
    multiset for_each_variant enumerates, for d = 1, 2."""
    rng = np.random.default_rng(21)
    for s in rand_seqs(rng, 600, 1, 26):
        for d in (1, 2):
            ref, _ = variants(hc, s, d)
            n = hc.hc_variant_count(s.encode(), len(s), d)
            buf = ctypes.create_string_buffer(19 * n)
            assert hc.hc_variants_flat(s.encode(), len(s), d, buf, n) == n
            flat = [buf.raw[19 * i : 19 * i + 19].split(b"\0")[0].decode() for i in range(n)]
            assert sorted(flat) == sorted(ref), (s, d)


def test_task_partition_of_variants(hc):
    """The staged scatter's balanced tasks cover every flat variant index exactly once."""
    rng = np.random.default_rng(23)
    for s in rand_seqs(rng, 2000, 1, 26):
        for d in (1, 2):
            assert hc.hc_task_variants_ok(s.encode(), len(s), d) == 1, (s, d)


def test_table_hashes_equal_variant_hashes(hc):
    """The key-table hashes of the d <= 2 kernels equal key_hash of each variant key."""
    rng = np.random.default_rng(29)
    for s in rand_seqs(rng, 1500, 1, 26) + ["A" * 30, "AAC" * 8, "ACACAC", "A", "AC"]:
        for d in (1, 2):
            assert hc.hc_table_hash_ok(s.encode(), len(s), d) == 1, (s, d)


def test_key_hash_definition(hc):
    """key_hash = finaliser(sum_k c_k r^k mod 2^64) over the first 18 residue codes."""
    M = (1 << 64) - 1
    r = 0x2545F4914F6CDD1D

    def fin(x):
        x ^= x >> 31
        x = (x * 0x9E3779B97F4A7C15) & M
        return x ^ (x >> 29)

    rng = np.random.default_rng(31)
    for s in rand_seqs(rng, 300, 1, 30):
        p = sum((ord(ch) - 64) * pow(r, k, 1 << 64) for k, ch in enumerate(s[:18])) & M
        assert hc.hc_key_hash(s.encode(), len(s)) == fin(p), s


def test_key_delete(hc):
    rng = np.random.default_rng(5)
    for s in rand_seqs(rng, 200, 1, 19):
        for p in range(len(s)):
            buf = ctypes.create_string_buffer(20)
            hc.hc_key_del(s.encode(), len(s), p, buf)
            assert buf.value.decode() == s[:p] + s[p + 1 :]


def test_levenshtein_myers_and_dp(hc):
    rng = np.random.default_rng(9)
    seqs = rand_seqs(rng, 400, 1, 70, "ACDEF")
    for a, b in zip(seqs[::2], seqs[1::2]):
        ref = orc.levenshtein(a, b)
        if len(a) <= 64:
            assert hc.hc_lev_myers(a.encode(), len(a), b.encode(), len(b)) == ref, (a, b)
        if len(a) <= 32:  # the 32-bit word form, patterns of up to 32 residues
            assert hc.hc_lev_myers32(a.encode(), len(a), b.encode(), len(b)) == ref, (a, b)
        assert hc.hc_lev_dp(a.encode(), len(a), b.encode(), len(b), 1000) == ref
        got = hc.hc_lev_dp(a.encode(), len(a), b.encode(), len(b), 2)
        assert (got == ref) if ref <= 2 else got > 2


def test_levenshtein_long(hc):
    rng = np.random.default_rng(10)
    for _ in range(20):
        a = "".join(rng.choice(list("ACD"), int(rng.integers(100, 500))))
        b = list(a)
        for _ in range(int(rng.integers(0, 4))):
            b[int(rng.integers(0, len(b)))] = "E"
        b = "".join(b)
        assert hc.hc_lev_dp(a.encode(), len(a), b.encode(), len(b), 1000) == orc.levenshtein(a, b)


def test_hamming_reference(hc):
    raw = ctypes.c_int()
    assert hc.hc_hamming(b"CAAA", 4, b"CAA", 3, ctypes.byref(raw)) == 77
    a, b = "A" * 200, "AC" * 100
    v = hc.hc_hamming(a.encode(), 200, b.encode(), 200, ctypes.byref(raw))
    assert raw.value == 100 and v == orc.hamming(a, b)
    a, b = "A" * 300, "C" * 300
    v = hc.hc_hamming(a.encode(), 300, b.encode(), 300, ctypes.byref(raw))
    assert raw.value == 300 and v == orc.hamming(a, b) == 44


def test_prefix_share_variant(hc):
    rng = np.random.default_rng(12)
    seqs = rand_seqs(rng, 600, 1, 24, "ACDE")
    for a, b in zip(seqs[::2], seqs[1::2]):
        for d in (1, 2, 3):
            va = set(orc.expand_keys(a, d))
            vb = set(orc.expand_keys(b, d))
            assert hc.hc_share_variant(a.encode(), len(a), b.encode(), len(b), d) == (1 if va & vb else 0), (a, b, d)


def test_triangle_rows(hc):
    for s in range(2, 40):
        l = 0
        for i in range(s - 1):
            assert hc.hc_tri_row_start(i, s) == l
            l += s - 1 - i


def test_hash_set_sizing(hc):
    """The candidate hash set's table sizes (the rule the engine applies; the sizes measured
    on B200 for the 1M and 10M workloads are the first two cases)."""
    first = hc.hc_dedup_first_table
    first.restype = ctypes.c_uint64
    first.argtypes = [ctypes.c_uint64, ctypes.c_double, ctypes.c_int]
    regrow = hc.hc_dedup_regrow_table
    regrow.restype = ctypes.c_uint64
    regrow.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
    # 1M: two slots per candidate fit in 256 MiB
    assert first(5_557_204, 1.0, 0) == 1 << 24
    assert first(5_557_204, 0.22, 0) == 1 << 24
    # 10M: above 256 MiB the previous search's distinct share sizes it (first search: all)
    assert first(55_000_000, 0.22, 0) == 1 << 25
    assert first(55_000_000, 1.0, 0) == 1 << 27
    # forced share sizing, with its 2^16-slot floor
    assert first(1000, 0.01, 1) == 1 << 16
    assert first(1_000_000, 0.5, 1) == 1 << 21
    for pc in (2, 1000, 1 << 20, 3_000_000, 40_000_000):
        for share in (0.01, 0.2, 0.8, 1.0):
            for forced in (0, 1):
                t = first(pc, share, forced)
                assert t & (t - 1) == 0 and t >= 2
                # at least two slots per expected distinct pair (1.25 x the share)
                assert t >= min(2 * pc, 2 * min(1.0, 1.25 * share) * pc)
    # a rerun gets four times the slots, and never fewer than two per candidate
    assert regrow(1 << 16, 1_000_000) == 1 << 21
    assert regrow(1 << 25, 1_000_000) == 1 << 27


def test_first_bad_offset_threaded_scan(hc):
    """The host length check of the whole-search entry point (first_bad_offset): from 2^20
    sequences on up to four threads scan parts of the offsets; the first bad sequence must be
    found wherever it lies (part boundaries, the last part) and with any thread count."""
    f = hc.hc_first_bad_offset
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    f.restype = ctypes.c_int
    n = (1 << 21) + 7
    lens = np.random.default_rng(12).integers(1, 40, n).astype(np.uint32)
    good = np.zeros(n + 1, np.uint32)
    good[1:] = np.cumsum(lens)
    for threads in (1, 2, 4):
        assert f(good.ctypes.data, n, threads) == -1
    for pos in (0, n // 4 - 1, n // 4, n // 2 + 3, 3 * n // 4, n - 1):
        for kind in ("empty", "long", "down"):
            o = good.copy()
            if kind == "empty":
                o[pos + 1:] -= lens[pos]  # sequence pos has no residues
            elif kind == "long":
                o[pos + 1:] += 501 - lens[pos]
            else:
                o[pos + 1] = o[pos] - 1 if o[pos] > 0 else 0
            for threads in (1, 2, 4):
                assert f(o.ctypes.data, n, threads) == pos, (pos, kind, threads)
    o = good.copy()
    o[n - 2 + 1:] += 600  # sequence n - 2 too long
    o[5 + 1:] -= lens[5]  # and sequence 5 empty: the first is reported
    assert f(o.ctypes.data, n, 4) == 5
    small = good[:1001].copy()
    small[11] = small[10]
    assert f(small.ctypes.data, 1000, 4) == 10
