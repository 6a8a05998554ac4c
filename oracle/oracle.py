"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker the CUDA product is compared against. It may be
loaded by the test suite, the smoke check and the benchmark's CPU-baseline leg, never by
the product. The functions restate the reference XTNeighbor-streaming path; see
oracle.cpp for the file:line each one follows.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_CLI = os.path.join(REF_DIR, "xt_neighbor_ref")
REF_HARNESS = os.path.join(REF_DIR, "ref_harness")

_lib = None
P = ctypes.c_void_p


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle not built: {LIB_PATH}")
        lib = ctypes.CDLL(LIB_PATH)
        lib.orc_expand_keys.restype = ctypes.c_int64
        lib.orc_stream1.restype = ctypes.c_int64
        lib.orc_stream3.restype = ctypes.c_int64
        lib.orc_stream4_nn.restype = ctypes.c_int64
        lib.orc_result_new.restype = P
        lib.orc_result_len.restype = ctypes.c_int64
        lib.orc_result_len.argtypes = [P]
        lib.orc_result_candidates.restype = ctypes.c_int64
        lib.orc_result_candidates.argtypes = [P]
        lib.orc_result_unique_candidates.restype = ctypes.c_int64
        lib.orc_result_unique_candidates.argtypes = [P]
        lib.orc_result_free.argtypes = [P]
        lib.orc_result_copy.argtypes = [P, P, P, P]
        lib.orc_nn_search.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        lib.orc_overlap_search.argtypes = [P, P, ctypes.c_int, P, ctypes.c_int, ctypes.c_int, P]
        lib.orc_brute_neighbors.restype = ctypes.c_int64
        lib.orc_brute_neighbors.argtypes = [P, P, ctypes.c_int, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P,
                                            ctypes.c_int64]
        _lib = lib
    return _lib


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(P)


def set_threads(n: int):
    load().orc_set_threads(int(n))


def threads() -> int:
    return load().orc_get_threads()


# ---------------------------------------------------------------- codec
def str_encode(s: str) -> np.ndarray:
    out = np.zeros(3, np.uint32)
    load().orc_str_encode(ctypes.c_char_p(s.encode()), ptr(out))
    return out


def str_decode(words) -> str:
    w = np.ascontiguousarray(words, dtype=np.uint32)
    buf = ctypes.create_string_buffer(20)
    load().orc_str_decode(ptr(w), buf)
    return buf.value.decode()


def len_decode(words) -> int:
    return load().orc_len_decode(ptr(np.ascontiguousarray(words, dtype=np.uint32)))


def remove_char(words, pos: int) -> np.ndarray:
    out = np.zeros(3, np.uint32)
    load().orc_remove_char(ptr(np.ascontiguousarray(words, dtype=np.uint32)), pos, ptr(out))
    return out


def char_encode(c: str) -> int:
    return load().orc_char_encode(ord(c))


def combination_len(words, d: int) -> int:
    return load().orc_combination_len(ptr(np.ascontiguousarray(words, dtype=np.uint32)), d)


def expand_keys(s: str, d: int) -> list[str]:
    """Deletion variants of str_encode(s) in the reference's DFS order."""
    w = str_encode(s)
    n = combination_len(w, d)
    out = np.zeros(3 * n, np.uint32)
    m = load().orc_expand_keys(ptr(w), d, ptr(out), None)
    return [str_decode(out[3 * i : 3 * i + 3]) for i in range(m)]


def expand_words(s: str, d: int) -> np.ndarray:
    w = str_encode(s)
    n = combination_len(w, d)
    out = np.zeros(3 * n, np.uint32)
    load().orc_expand_keys(ptr(w), d, ptr(out), None)
    return out.reshape(-1, 3)


# ---------------------------------------------------------------- stages
def stream1(seqs: list[str], d: int, nbins: int, carry: int = 0):
    keys = np.stack([str_encode(s) for s in seqs]).astype(np.uint32)
    total = sum(combination_len(k, d) for k in keys)
    kout = np.zeros(3 * total, np.uint32)
    ids = np.zeros(total, np.int32)
    hist = np.zeros(nbins, np.int32)
    n = load().orc_stream1(ptr(keys), len(seqs), d, carry, nbins, ptr(kout), ptr(ids), ptr(hist))
    return [str_decode(kout[3 * i : 3 * i + 3]) for i in range(n)], ids[:n], hist


def stream2(keys: list[str], ids, seq_len: int, nbins: int, max_row: int):
    k = np.stack([str_encode(s) for s in keys]).astype(np.uint32)
    v = np.ascontiguousarray(ids, dtype=np.int32)
    hist = np.zeros(nbins, np.int32)
    rows = np.zeros(len(keys) + 1, np.int32)
    nr = load().orc_stream2(ptr(k), ptr(v), len(keys), seq_len, nbins, max_row, ptr(hist), ptr(rows))
    return [str_decode(k[i]) for i in range(len(keys))], v, hist, rows[:nr]


def stream3(keys: list[str], ids, lowerbound: int, seq_len: int, nbins: int):
    k = np.stack([str_encode(s) for s in keys]).astype(np.uint32)
    v = np.ascontiguousarray(ids, dtype=np.int32).copy()
    n = ctypes.c_int(len(keys))
    cap = len(keys) * len(keys)
    pairs = np.zeros(2 * cap, np.int32)
    hist = np.zeros(nbins, np.int32)
    np_ = load().orc_stream3(ptr(k), ptr(v), ctypes.byref(n), lowerbound, seq_len, nbins, ptr(pairs), ctypes.c_int64(cap), ptr(hist))
    m = n.value
    return pairs[: 2 * np_].reshape(-1, 2), hist, [str_decode(k[i]) for i in range(m)], v[:m]


def stream4_nn(chars, offs, seq_len: int, pairs, d: int, measure: int):
    pr = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1)
    n = len(pr) // 2
    out = np.zeros(2 * max(n, 1), np.int32)
    dist = np.zeros(max(n, 1), np.int8)
    m = load().orc_stream4_nn(ptr(chars), ptr(offs), seq_len, ptr(pr), ctypes.c_int64(n), d, measure, ptr(out), ptr(dist))
    return out[: 2 * m].reshape(-1, 2), dist[:m]


def histogram(values, nbins: int, lo: int, hi: int) -> np.ndarray:
    v = np.ascontiguousarray(values, dtype=np.int32)
    out = np.zeros(nbins, np.int32)
    load().orc_histogram_i32(ptr(v), ctypes.c_int64(len(v)), nbins, ctypes.c_int64(lo), ctypes.c_int64(hi), ptr(out))
    return out


def bin_packing_offsets(hist, exponent: int):
    h = np.ascontiguousarray(hist, dtype=np.int32)
    nrow, nlevel = h.shape
    out = np.zeros(nrow * nlevel + 1, np.int32)
    per = load().orc_bin_packing_offsets(ptr(h), nrow, nlevel, exponent, ptr(out))
    return per, out[: per * nrow].reshape(nrow, per) if per > 0 else None


def bin_packing_lowerbounds(hist, seq_len: int, exponent: int):
    h = np.ascontiguousarray(hist, dtype=np.int32)
    nrow, nlevel = h.shape
    out = np.zeros(nlevel, np.int32)
    n = load().orc_bin_packing_lowerbounds(ptr(h), nrow, nlevel, seq_len, exponent, ptr(out))
    return out[:n]


def overlap_init(chars, offs, info):
    inf = np.ascontiguousarray(info, dtype=np.int32).reshape(-1, 3).copy()
    n = len(inf)
    cum = np.zeros(n, np.int32)
    keys = np.zeros(3 * n, np.uint32)
    dp = np.zeros(2 * n * n + 2, np.int32)
    ds = np.zeros(n * n + 1, np.uint64)
    nd = ctypes.c_int(0)
    u = load().orc_overlap_init(ptr(chars), ptr(offs), ptr(inf), n, ptr(cum), ptr(keys), ptr(dp), ptr(ds), ctypes.byref(nd))
    m = nd.value
    return u, inf, cum[:u], keys[: 3 * u].reshape(-1, 3), dp[: 2 * m].reshape(-1, 2), ds[:m]


def stream4_overlap(chars, offs, info_sorted, cum_counts, pairs, d: int, measure: int):
    inf = np.ascontiguousarray(info_sorted, dtype=np.int32).reshape(-1)
    cum = np.ascontiguousarray(cum_counts, dtype=np.int32)
    pr = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1)
    cap = 4096
    rp = np.zeros(2 * cap, np.int32)
    sums = np.zeros(cap, np.uint64)
    m = load().orc_stream4_overlap(ptr(chars), ptr(offs), ptr(inf), ptr(cum), len(cum), ptr(pr), ctypes.c_int64(len(pr) // 2), d, measure, ptr(rp), ptr(sums))
    return rp[: 2 * m].reshape(-1, 2), sums[:m]


# ---------------------------------------------------------------- whole searches
def nn_search(chars, offs, d: int, measure: int = 0):
    """Sorted (x, y) pairs, int8 distances and candidate counts of the reference algorithm."""
    lib = load()
    chars = np.ascontiguousarray(chars, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.uint32)
    r = lib.orc_result_new()
    try:
        lib.orc_nn_search(ptr(chars), ptr(offs), len(offs) - 1, d, measure, r)
        m = lib.orc_result_len(r)
        pairs = np.zeros((m, 2), np.int32)
        dist = np.zeros(m, np.int8)
        lib.orc_result_copy(r, ptr(pairs), ptr(dist), None)
        meta = {"candidates": lib.orc_result_candidates(r), "unique": lib.orc_result_unique_candidates(r)}
        return pairs, dist, meta
    finally:
        lib.orc_result_free(r)


def overlap_search(chars, offs, info, d: int, measure: int = 0):
    """Sorted (rep_x, rep_y) entries with their uint64 sums."""
    lib = load()
    chars = np.ascontiguousarray(chars, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.uint32)
    inf = np.ascontiguousarray(info, dtype=np.int32).reshape(-1, 3)
    r = lib.orc_result_new()
    try:
        lib.orc_overlap_search(ptr(chars), ptr(offs), len(offs) - 1, ptr(inf), d, measure, r)
        m = lib.orc_result_len(r)
        pairs = np.zeros((m, 2), np.int32)
        sums = np.zeros(m, np.uint64)
        lib.orc_result_copy(r, ptr(pairs), None, ptr(sums))
        return pairs, sums
    finally:
        lib.orc_result_free(r)


def brute_neighbors(chars, offs, queries, d: int, measure: int = 0):
    """Exhaustive (min, max, dist) neighbours of the query sequences, sorted; equal to the
    reference output restricted to those queries for sequences shorter than 128 residues."""
    lib = load()
    chars = np.ascontiguousarray(chars, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.uint32)
    q = np.ascontiguousarray(queries, dtype=np.int32)
    cap = 1 << 16
    while True:
        out = np.zeros(3 * cap, np.int32)
        m = lib.orc_brute_neighbors(ptr(chars), ptr(offs), len(offs) - 1, ptr(q), len(q), d, measure, ptr(out), cap)
        if m <= cap:
            return out[: 3 * m].reshape(-1, 3)
        cap = int(m)


def levenshtein(a: str, b: str) -> int:
    return load().orc_levenshtein(a.encode(), len(a), b.encode(), len(b))


def hamming(a: str, b: str) -> int:
    return load().orc_hamming(a.encode(), len(a), b.encode(), len(b))
