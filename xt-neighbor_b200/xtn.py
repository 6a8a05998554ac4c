"""ctypes binding of the xtn_b200 C ABI (include/xtn_b200.h).

This is the Python mirror of the reference's library entry point
``xtn_perform(XTNArgs, SeqArray*, SeqInfo*, callback)`` (xtneighbor_streaming/src/xtn.cu:267):
``Context.perform`` takes the CSR sequence store the reference's SeqArray holds, an optional
per-row SeqInfo table (overlap mode) and returns the concatenated XTNOutput chunks.
The compute path is the CUDA library ``lib/libxtn_b200.so``; there is no CPU fallback:
loading fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("XTN_LIB") or os.path.join(HERE, "lib", "libxtn_b200.so")
SYNTH_PATH = os.path.join(HERE, "lib", "libxtn_synth.so")
CLI_PATH = os.path.join(HERE, "bin", "xt_neighbor")

LEVENSHTEIN = 0  # xtneighbor_streaming/src/xtn.h:12
HAMMING = 1  # xtneighbor_streaming/src/xtn.h:14

SUCCESS, ERROR, EXIT = 0, 1, 2
ERR_CUDA, ERR_NOMEM, ERR_ARG, ERR_NODEV, ERR_LIMIT = 3, 4, 5, 6, 7

SYMBOLS = (
    "xtn_perform",
    "xtn_context_create",
    "xtn_context_destroy",
    "xtn_context_perform",
    "xtn_context_nn_device",
    "xtn_context_overlap_device",
    "xtn_index_create",
    "xtn_index_create_device",
    "xtn_index_destroy",
    "xtn_index_stats",
    "xtn_index_context",
    "xtn_index_query",
    "xtn_index_query_device",
    "xtn_index_serve",
    "xtn_context_fetch",
    "xtn_context_result_device",
    "xtn_context_result_keys",
    "xtn_context_merge_keys",
    "xtn_shard_generate",
    "xtn_shard_search",
    "xtn_context_stream",
    "xtn_context_stats",
    "xtn_context_set_option",
    "xtn_context_autotune",
    "xtn_context_set_profiling",
    "xtn_context_kernel_times",
    "xtn_context_profile_only",
    "xtn_last_error",
    "xtn_version",
)


class Int2(ctypes.Structure):
    _fields_ = [("x", ctypes.c_int32), ("y", ctypes.c_int32)]


class SeqInfo(ctypes.Structure):
    _fields_ = [("frequency", ctypes.c_int32), ("repertoire", ctypes.c_int32), ("original_index", ctypes.c_int32)]


class Args(ctypes.Structure):
    _fields_ = [
        ("distance", ctypes.c_int32),
        ("measure", ctypes.c_int32),
        ("verbose", ctypes.c_int32),
        ("info_len", ctypes.c_int32),
    ]


class Output(ctypes.Structure):
    _fields_ = [
        ("index_pairs", ctypes.POINTER(Int2)),
        ("pairwise_distances", ctypes.POINTER(ctypes.c_int8)),
        ("pairwise_frequencies", ctypes.POINTER(ctypes.c_uint64)),
        ("len", ctypes.c_int64),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_seqs", ctypes.c_int64),
        ("n_variants", ctypes.c_int64),
        ("n_groups", ctypes.c_int64),
        ("n_candidates", ctypes.c_int64),
        ("n_unique", ctypes.c_int64),
        ("n_out", ctypes.c_int64),
        ("n_verified_pairs", ctypes.c_int64),
        ("n_launches", ctypes.c_int64),
        ("id_bits", ctypes.c_int32),
        ("n_rounds", ctypes.c_int32),
        ("ms_total", ctypes.c_double),
        ("ms_stage", ctypes.c_double * 8),
        ("n_fallback", ctypes.c_int64),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "ms_stage"}
        d["ms_stage"] = list(self.ms_stage)
        return d


CALLBACK = ctypes.CFUNCTYPE(None, ctypes.POINTER(Output), ctypes.c_void_p)


class IndexInfo(ctypes.Structure):
    _fields_ = [
        ("n_seqs", ctypes.c_int64),
        ("n_records", ctypes.c_int64),
        ("bytes", ctypes.c_int64),
        ("max_distance", ctypes.c_int32),
        ("directory_bits", ctypes.c_int32),
        ("ms_build", ctypes.c_double),
    ]


class Request(ctypes.Structure):
    _fields_ = [
        ("seqs", ctypes.c_void_p),
        ("offsets", ctypes.c_void_p),
        ("n_seqs", ctypes.c_int32),
        ("distance", ctypes.c_int32),
        ("measure", ctypes.c_int32),
        ("arrival_s", ctypes.c_double),
    ]


class RequestResult(ctypes.Structure):
    _fields_ = [
        ("admitted_s", ctypes.c_double),
        ("done_s", ctypes.c_double),
        ("n_out", ctypes.c_int64),
        ("batch", ctypes.c_int32),
        ("status", ctypes.c_int32),
    ]


class ServeOptions(ctypes.Structure):
    _fields_ = [("max_batch_seqs", ctypes.c_int64), ("hbm_fraction", ctypes.c_double), ("realtime", ctypes.c_int32),
                ("slots", ctypes.c_int32)]


REQUEST_CALLBACK = ctypes.CFUNCTYPE(None, ctypes.c_int32, ctypes.POINTER(Output), ctypes.c_void_p)

_lib = None


class XtnError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"xtn_b200 error {code}: {msg}")
        self.code = code


def load():
    """Loads lib/libxtn_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library not built: {LIB_PATH} is missing (run __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    lib.xtn_last_error.restype = ctypes.c_char_p
    lib.xtn_version.restype = ctypes.c_char_p
    lib.xtn_context_create.argtypes = [ctypes.c_int, ctypes.POINTER(P)]
    lib.xtn_context_destroy.argtypes = [P]
    lib.xtn_context_destroy.restype = None
    lib.xtn_context_perform.argtypes = [P, ctypes.POINTER(Args), P, P, ctypes.c_int32, P, CALLBACK, P]
    lib.xtn_perform.argtypes = [ctypes.POINTER(Args), P, P, ctypes.c_int32, P, CALLBACK, P]
    lib.xtn_context_nn_device.argtypes = [P, ctypes.POINTER(Args), P, P, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]
    lib.xtn_context_overlap_device.argtypes = [P, ctypes.POINTER(Args), P, P, ctypes.c_int32, P,
                                               ctypes.POINTER(ctypes.c_int64)]
    lib.xtn_context_fetch.argtypes = [P, P, P, P, ctypes.c_int64]
    lib.xtn_context_autotune.argtypes = [P, ctypes.POINTER(Args), P, P, ctypes.c_int32, ctypes.c_int32, P,
                                         ctypes.c_int32]
    lib.xtn_index_create.argtypes = [ctypes.c_int, P, P, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(P)]
    lib.xtn_index_create_device.argtypes = [ctypes.c_int, P, P, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(P)]
    lib.xtn_index_destroy.argtypes = [P]
    lib.xtn_index_destroy.restype = None
    lib.xtn_index_stats.argtypes = [P, ctypes.POINTER(IndexInfo)]
    lib.xtn_index_context.argtypes = [P]
    lib.xtn_index_context.restype = P
    lib.xtn_index_query.argtypes = [P, ctypes.POINTER(Args), P, P, ctypes.c_int32, CALLBACK, P]
    lib.xtn_index_query_device.argtypes = [P, ctypes.POINTER(Args), P, P, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]
    lib.xtn_index_serve.argtypes = [P, ctypes.POINTER(Request), ctypes.c_int32, ctypes.POINTER(ServeOptions),
                                    ctypes.POINTER(RequestResult), REQUEST_CALLBACK, P]
    lib.xtn_context_result_device.argtypes = [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(ctypes.c_int64)]
    lib.xtn_context_result_keys.argtypes = [P, ctypes.c_int32, P, ctypes.c_int64, ctypes.c_int32,
                                            ctypes.POINTER(ctypes.c_int64)]
    lib.xtn_context_merge_keys.argtypes = [P, ctypes.c_int32, P, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    lib.xtn_shard_generate.argtypes = [P, ctypes.POINTER(Args), P, P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                       P, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(P),
                                       ctypes.POINTER(ctypes.c_int64)]
    lib.xtn_shard_search.argtypes = [P, ctypes.POINTER(Args), P, P, ctypes.c_int32, P, P, ctypes.c_int32,
                                     ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]
    lib.xtn_context_stream.argtypes = [P]
    lib.xtn_context_stream.restype = P
    lib.xtn_context_stats.argtypes = [P, ctypes.POINTER(Stats)]
    lib.xtn_context_set_profiling.argtypes = [P, ctypes.c_int]
    lib.xtn_context_profile_only.argtypes = [P, ctypes.c_char_p]
    lib.xtn_context_set_option.argtypes = [P, ctypes.c_char_p, ctypes.c_int64]
    lib.xtn_context_kernel_times.argtypes = [P, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
    _lib = lib
    return lib


def _check(code: int):
    if code != SUCCESS:
        raise XtnError(code, load().xtn_last_error().decode(errors="replace"))


def pack_sequences(seqs) -> tuple[np.ndarray, np.ndarray]:
    """List of strings -> (chars uint8, offsets uint32) CSR store, as SeqArray keeps it."""
    enc = [s.encode() for s in seqs]
    offs = np.zeros(len(enc) + 1, dtype=np.uint32)
    if enc:
        offs[1:] = np.cumsum([len(e) for e in enc])
    chars = np.frombuffer(b"".join(enc), dtype=np.uint8).copy()
    return chars, offs


def unpack_sequences(chars: np.ndarray, offs: np.ndarray) -> list[str]:
    b = chars.tobytes()
    return [b[offs[i] : offs[i + 1]].decode() for i in range(len(offs) - 1)]


@dataclass
class Result:
    pairs: np.ndarray  # (n, 2) int32
    distances: np.ndarray | None  # (n,) int8, NN mode
    frequencies: np.ndarray | None  # (n,) uint64, overlap mode


class Context:
    """Reusable device context (stream + growing device buffers)."""

    def __init__(self, device: int = 0, **options):
        self.lib = load()
        self.h = ctypes.c_void_p()
        _check(self.lib.xtn_context_create(device, ctypes.byref(self.h)))
        for k, v in options.items():
            self.set_option(k, v)

    def set_option(self, name: str, value: int):
        _check(self.lib.xtn_context_set_option(self.h, name.encode(), int(value)))

    def close(self):
        if self.h:
            self.lib.xtn_context_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def perform(self, chars, offsets, distance=1, measure=LEVENSHTEIN, info=None, n_reps=0, verbose=0) -> Result:
        """The whole search on host buffers (xtn_context_perform)."""
        chars = np.ascontiguousarray(chars, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        n = len(offsets) - 1
        args = Args(distance, measure, verbose, n_reps)
        chunks_p, chunks_v = [], []
        overlap = info is not None

        def cb(out_ptr, _user):
            o = out_ptr.contents
            m = o.len
            if m <= 0:
                return
            pp = ctypes.cast(o.index_pairs, ctypes.POINTER(ctypes.c_int32))
            chunks_p.append(np.ctypeslib.as_array(pp, shape=(m, 2)).copy())
            if overlap:
                chunks_v.append(np.ctypeslib.as_array(o.pairwise_frequencies, shape=(m,)).copy())
            else:
                chunks_v.append(np.ctypeslib.as_array(o.pairwise_distances, shape=(m,)).copy())

        ccb = CALLBACK(cb)
        info_arr = None
        if overlap:
            info_arr = np.ascontiguousarray(info, dtype=np.int32).reshape(-1, 3)
        rc = self.lib.xtn_context_perform(
            self.h,
            ctypes.byref(args),
            chars.ctypes.data_as(ctypes.c_void_p),
            offsets.ctypes.data_as(ctypes.c_void_p),
            n,
            info_arr.ctypes.data_as(ctypes.c_void_p) if overlap else None,
            ccb,
            None,
        )
        _check(rc)

        def joined(chunks, empty):
            if not chunks:
                return empty
            return chunks[0] if len(chunks) == 1 else np.concatenate(chunks)

        pairs = joined(chunks_p, np.zeros((0, 2), np.int32))
        if overlap:
            return Result(pairs, None, joined(chunks_v, np.zeros(0, np.uint64)))
        return Result(pairs, joined(chunks_v, np.zeros(0, np.int8)), None)

    def nn_device(self, d_chars: int, d_offsets: int, n: int, distance=1, measure=LEVENSHTEIN) -> int:
        """Search on device pointers; returns the number of output pairs (kept on device)."""
        args = Args(distance, measure, 0, 0)
        nout = ctypes.c_int64()
        _check(
            self.lib.xtn_context_nn_device(
                self.h, ctypes.byref(args), ctypes.c_void_p(d_chars), ctypes.c_void_p(d_offsets), n, ctypes.byref(nout)
            )
        )
        return nout.value

    def overlap_device(self, d_chars: int, d_offsets: int, n: int, d_info: int, n_reps: int, distance=1,
                       measure=LEVENSHTEIN) -> int:
        """Overlap mode on device pointers (d_info: n x 3 int32 rows of frequency, repertoire,
        original index); returns the number of (rep_x, rep_y) entries (kept on device)."""
        args = Args(distance, measure, 0, n_reps)
        nout = ctypes.c_int64()
        _check(
            self.lib.xtn_context_overlap_device(
                self.h, ctypes.byref(args), ctypes.c_void_p(d_chars), ctypes.c_void_p(d_offsets), n,
                ctypes.c_void_p(d_info), ctypes.byref(nout)
            )
        )
        return nout.value

    def fetch_overlap(self, n: int) -> Result:
        pairs = np.zeros((n, 2), np.int32)
        sums = np.zeros(n, np.uint64)
        _check(
            self.lib.xtn_context_fetch(
                self.h, pairs.ctypes.data_as(ctypes.c_void_p), None, sums.ctypes.data_as(ctypes.c_void_p), n
            )
        )
        return Result(pairs, None, sums)

    def autotune(self, d_chars: int, d_offsets: int, n: int, distance=1, measure=LEVENSHTEIN, repeats=2) -> str:
        """Times the bucket engine's shapes on these device inputs and keeps the fastest on the
        context (xtn_context_autotune); returns the choice as text."""
        args = Args(distance, measure, 0, 0)
        buf = ctypes.create_string_buffer(256)
        _check(self.lib.xtn_context_autotune(self.h, ctypes.byref(args), ctypes.c_void_p(d_chars),
                                             ctypes.c_void_p(d_offsets), n, repeats, buf, 256))
        return buf.value.decode()

    def fetch(self, n: int) -> Result:
        pairs = np.zeros((n, 2), np.int32)
        dist = np.zeros(n, np.int8)
        _check(
            self.lib.xtn_context_fetch(
                self.h, pairs.ctypes.data_as(ctypes.c_void_p), dist.ctypes.data_as(ctypes.c_void_p), None, n
            )
        )
        return Result(pairs, dist, None)

    def stream(self) -> int:
        return self.lib.xtn_context_stream(self.h) or 0

    def result_keys(self, n: int, d_keys: int, capacity: int, n_ranges: int) -> list:
        """Writes the last result as 64-bit pair keys to d_keys (xtn_context_result_keys) and
        returns the n_ranges + 1 range starts by owner rank."""
        starts = (ctypes.c_int64 * (n_ranges + 1))()
        _check(self.lib.xtn_context_result_keys(self.h, n, ctypes.c_void_p(d_keys), capacity, n_ranges, starts))
        return list(starts)

    def shard_generate(self, d_chars: int, d_offsets: int, n: int, distance: int, measure: int, rank: int,
                       n_ranks: int):
        """xtn_shard_generate: this rank's variant records in the search's first-level buckets.
        Returns (per-bucket counts as uint64 array, device pointer of the records, record count)."""
        args = Args(distance, measure, 0, 0)
        cap = 1 << 15
        counts = np.zeros(cap, np.uint64)
        nb = ctypes.c_int32()
        ptr = ctypes.c_void_p()
        nrec = ctypes.c_int64()
        _check(self.lib.xtn_shard_generate(self.h, ctypes.byref(args), ctypes.c_void_p(d_chars),
                                           ctypes.c_void_p(d_offsets), n, rank, n_ranks,
                                           counts.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(nb),
                                           ctypes.byref(ptr), ctypes.byref(nrec)))
        return counts[: nb.value].copy(), ptr.value or 0, nrec.value

    def shard_search(self, d_chars: int, d_offsets: int, n: int, distance: int, measure: int, d_records: int,
                     piece_counts) -> int:
        """xtn_shard_search over the pieces a rank received (piece_counts: n_pieces x b_n)."""
        args = Args(distance, measure, 0, 0)
        pc = np.ascontiguousarray(piece_counts, dtype=np.uint64)
        nout = ctypes.c_int64()
        _check(self.lib.xtn_shard_search(self.h, ctypes.byref(args), ctypes.c_void_p(d_chars),
                                         ctypes.c_void_p(d_offsets), n, ctypes.c_void_p(d_records),
                                         pc.ctypes.data_as(ctypes.c_void_p), pc.shape[0], pc.shape[1],
                                         ctypes.byref(nout)))
        return nout.value

    def merge_keys(self, n: int, d_keys: int, count: int) -> int:
        """Sorts and de-duplicates received pair keys into the context's result
        (xtn_context_merge_keys); returns its length."""
        nout = ctypes.c_int64()
        _check(self.lib.xtn_context_merge_keys(self.h, n, ctypes.c_void_p(d_keys), count, ctypes.byref(nout)))
        return nout.value

    def set_profiling(self, on: bool, only: str = None):
        """Brackets kernel launches with CUDA events; `only` restricts that to one kernel name."""
        _check(self.lib.xtn_context_set_profiling(self.h, 1 if on else 0))
        _check(self.lib.xtn_context_profile_only(self.h, only.encode() if only else None))

    def kernel_times(self) -> dict:
        """{kernel name: (total ms, launches)} of the last run (profiling on)."""
        cap = 64
        names = (ctypes.c_char_p * cap)()
        ms = (ctypes.c_double * cap)()
        ln = (ctypes.c_int64 * cap)()
        n = self.lib.xtn_context_kernel_times(self.h, names, ms, ln, cap)
        return {names[i].decode(): (ms[i], ln[i]) for i in range(min(n, cap))}

    def stats(self) -> dict:
        st = Stats()
        _check(self.lib.xtn_context_stats(self.h, ctypes.byref(st)))
        return st.as_dict()


# ---------------------------------------------------------------- synthetic data (host)
_synth = None


def _load_synth():
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_PATH):
            raise RuntimeError(f"generator library not built: {SYNTH_PATH}")
        s = ctypes.CDLL(SYNTH_PATH)
        s.synth_nn.restype = ctypes.c_void_p
        s.synth_nn.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        s.synth_overlap.restype = ctypes.c_void_p
        s.synth_overlap.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        for f in ("synth_n", "synth_total_chars"):
            getattr(s, f).restype = ctypes.c_int64
            getattr(s, f).argtypes = [ctypes.c_void_p]
        s.synth_n_reps.restype = ctypes.c_int32
        s.synth_n_reps.argtypes = [ctypes.c_void_p]
        s.synth_copy.argtypes = [ctypes.c_void_p] * 5
        s.synth_free.argtypes = [ctypes.c_void_p]
        _synth = s
    return _synth


def _take(h, with_info=False):
    s = _load_synth()
    n, nc, nr = s.synth_n(h), s.synth_total_chars(h), s.synth_n_reps(h)
    chars = np.zeros(nc, np.uint8)
    offs = np.zeros(n + 1, np.uint32)
    freq = np.zeros(n if with_info else 0, np.int32)
    reps = np.zeros(nr, np.int32)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a.size else None
    s.synth_copy(h, ptr(chars), ptr(offs), ptr(freq), ptr(reps))
    s.synth_free(h)
    return chars, offs, freq, reps


def synth_mutants(seed: int, n: int, mutant_frac: float = 0.10):
    """n generator sequences, a fraction of them 1-2 edit mutants of earlier rows."""
    chars, offs, _, _ = _take(_load_synth().synth_nn(seed, n, 0, mutant_frac, 0.0))
    return chars, offs


def synth_clusters(seed: int, n: int, cluster_frac: float = 0.20, dup_frac: float = 0.02):
    """n generator sequences with mutant clusters and exact duplicates, shuffled."""
    chars, offs, _, _ = _take(_load_synth().synth_nn(seed, n, 1, cluster_frac, dup_frac))
    return chars, offs


def exchange_keys(keys, starts, group=None):
    """All-to-all of pair keys by owner rank (torch.distributed, NCCL for CUDA tensors, gloo on
    CPU): keys[starts[k]:starts[k+1]] go to rank k; returns what this rank receives (the
    sources' runs in rank order). Sizes are exchanged first, so every rank takes the same two
    collective steps."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    send = [int(starts[k + 1] - starts[k]) for k in range(world)]
    sizes = torch.tensor(send, dtype=torch.int64, device=keys.device)
    got = torch.empty(world, dtype=torch.int64, device=keys.device)
    dist.all_to_all_single(got, sizes, group=group)
    recv = [int(v) for v in got.tolist()]
    out = torch.empty(sum(recv), dtype=torch.int64, device=keys.device)
    dist.all_to_all_single(out, keys[: starts[world]].contiguous(), recv, send, group=group)
    return out


class _DeviceWords:
    """A view of n int64 words of device memory for torch.as_tensor (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i8", "data": (ptr, False), "version": 3}


def owner_ranges(counts, n_ranks: int):
    """First-level buckets of each rank: rank k owns [bounds[k], bounds[k + 1]), contiguous
    ranges that start at the bucket holding record k V / K of the V records (the same rule as
    the shard_count option's)."""
    counts = np.asarray(counts, dtype=np.int64)
    starts = np.concatenate([[0], np.cumsum(counts)])
    total = int(starts[-1])
    nb = len(counts)
    bounds = [0]
    for k in range(1, n_ranks):
        b = int(np.searchsorted(starts[:nb], total * k // n_ranks, side="left"))
        bounds.append(max(bounds[-1], b))
    bounds.append(nb)
    return bounds


def exchange_records(counts, recs, group=None):
    """The record exchange of a sequence-sharded search: this rank's records `recs` (int64, on
    the device the collectives use), partitioned into the search's first-level buckets with
    counts[b] records in bucket b, go to the ranks that own their buckets. The bucket counts
    are summed over the ranks (all-reduce), rank k owns owner_ranges(totals, K)[k:k+2], and two
    all-to-alls send each owner its buckets' records and their per-bucket counts. Returns (the
    records this rank received, one piece per source rank in rank order; piece_counts, a
    K x b_n uint64 array: piece p holds piece_counts[p, j] records of this rank's j-th bucket;
    the owner bounds)."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    local = torch.from_numpy(np.asarray(counts).astype(np.int64)).to(recs.device)
    total = local.clone()
    dist.all_reduce(total, group=group)
    bounds = owner_ranges(total.cpu().numpy(), world)
    cum = np.concatenate([[0], np.cumsum(np.asarray(counts).astype(np.int64))])
    # records: keys [cum[bounds[k]], cum[bounds[k+1]]) go to rank k
    got = exchange_keys(recs, [int(cum[b]) for b in bounds], group)
    # per-bucket counts of the sent pieces: counts[bounds[k]:bounds[k+1]] go to rank k
    got_counts = exchange_keys(local, bounds, group)
    b_n = bounds[rank + 1] - bounds[rank]
    piece_counts = got_counts.cpu().numpy().astype(np.uint64).reshape(world, b_n)
    return got, piece_counts, bounds


def nn_sharded_exchange(ctx, d_chars: int, d_offsets: int, n: int, distance=1, measure=LEVENSHTEIN,
                        group=None) -> int:
    """One rank's part of a search sharded by sequences (xtn_shard_generate / xtn_shard_search):
    every rank generates its own sequences' variant records in the first-level buckets; the
    bucket counts are summed over the ranks, each rank gets a contiguous range of buckets, and
    two all-to-alls send it its buckets' per-source counts and records; the rank then searches
    its buckets, and the verified pairs are exchanged by owner and merged as in nn_sharded.
    Returns the number of pairs left as the context's result (this rank's id range)."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device())
    counts, ptr, nrec = ctx.shard_generate(d_chars, d_offsets, n, distance, measure, rank, world)
    recs = torch.as_tensor(_DeviceWords(ptr, nrec), device=dev) if nrec > 0 else torch.zeros(1, dtype=torch.int64,
                                                                                             device=dev)
    got, piece_counts, _ = exchange_records(counts, recs, group)
    m = ctx.shard_search(d_chars, d_offsets, n, distance, measure, got.data_ptr(), piece_counts)
    keys = torch.empty(max(m, 1), dtype=torch.int64, device=dev)
    starts = ctx.result_keys(n, keys.data_ptr(), keys.numel(), world)
    merged = exchange_keys(keys, starts, group)
    return ctx.merge_keys(n, merged.data_ptr(), merged.numel())


def nn_sharded(ctx, d_chars: int, d_offsets: int, n: int, distance=1, measure=LEVENSHTEIN, group=None) -> int:
    """One rank's part of a nearest-neighbour search sharded over the ranks of `group` (one GPU
    each, the same input on every rank): the search over this rank's share of the first-level
    hash buckets (context options shard_count / shard_index), the exchange of the verified pairs
    by owner (pairs whose x lies in this rank's id range come here), and the merge. Returns the
    number of pairs left as the context's result: this rank's id range of the whole output, in
    order, so that the ranks' results in rank order are the unsharded search's output."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    ctx.set_option("shard_count", world)
    ctx.set_option("shard_index", rank)
    m = ctx.nn_device(d_chars, d_offsets, n, distance, measure)
    dev = torch.device("cuda", torch.cuda.current_device())
    keys = torch.empty(max(m, 1), dtype=torch.int64, device=dev)
    starts = ctx.result_keys(n, keys.data_ptr(), keys.numel(), world)
    got = exchange_keys(keys, starts, group)
    return ctx.merge_keys(n, got.data_ptr(), got.numel())


def synth_repertoires(seed: int, n_reps: int, min_size: float, max_size: float, shared: float = 0.05):
    """Repertoire-overlap input: (chars, offsets, info (n,3) int32, rep_sizes)."""
    chars, offs, freq, reps = _take(_load_synth().synth_overlap(seed, n_reps, min_size, max_size, shared), True)
    n = len(offs) - 1
    rep_of = np.repeat(np.arange(len(reps), dtype=np.int32), reps)
    info = np.stack([freq, rep_of, np.arange(n, dtype=np.int32)], axis=1).astype(np.int32)
    return chars, offs, info, reps


class Index:
    """Resident deletion index over reference sequences (xtn_index_*): query batches return the
    (index row, n_index + batch row) pairs the offline search would report on the union."""

    def __init__(self, chars, offsets, max_distance: int = 2, device: int = 0):
        self.lib = load()
        self.h = ctypes.c_void_p()
        chars = np.ascontiguousarray(chars, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        self.n = len(offsets) - 1
        _check(self.lib.xtn_index_create(device, chars.ctypes.data_as(ctypes.c_void_p),
                                         offsets.ctypes.data_as(ctypes.c_void_p), self.n, max_distance,
                                         ctypes.byref(self.h)))
        self.ctx = Context.__new__(Context)
        self.ctx.lib = self.lib
        self.ctx.h = ctypes.c_void_p(self.lib.xtn_index_context(self.h))

    def close(self):
        if self.h:
            self.lib.xtn_index_destroy(self.h)
            self.h = ctypes.c_void_p()
            self.ctx.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def info(self) -> dict:
        st = IndexInfo()
        _check(self.lib.xtn_index_stats(self.h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def query(self, chars, offsets, distance=1, measure=LEVENSHTEIN) -> Result:
        chars = np.ascontiguousarray(chars, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        args = Args(distance, measure, 0, 0)
        chunks_p, chunks_d = [], []

        def cb(out_ptr, _user):
            o = out_ptr.contents
            if o.len <= 0:
                return
            pp = ctypes.cast(o.index_pairs, ctypes.POINTER(ctypes.c_int32))
            chunks_p.append(np.ctypeslib.as_array(pp, shape=(o.len, 2)).copy())
            chunks_d.append(np.ctypeslib.as_array(o.pairwise_distances, shape=(o.len,)).copy())

        ccb = CALLBACK(cb)
        _check(self.lib.xtn_index_query(self.h, ctypes.byref(args), chars.ctypes.data_as(ctypes.c_void_p),
                                        offsets.ctypes.data_as(ctypes.c_void_p), len(offsets) - 1, ccb, None))
        pairs = np.concatenate(chunks_p) if chunks_p else np.zeros((0, 2), np.int32)
        dist = np.concatenate(chunks_d) if chunks_d else np.zeros(0, np.int8)
        return Result(pairs, dist, None)

    def query_device(self, d_chars: int, d_offsets: int, n: int, distance=1, measure=LEVENSHTEIN) -> int:
        args = Args(distance, measure, 0, 0)
        nout = ctypes.c_int64()
        _check(self.lib.xtn_index_query_device(self.h, ctypes.byref(args), ctypes.c_void_p(d_chars),
                                               ctypes.c_void_p(d_offsets), n, ctypes.byref(nout)))
        return nout.value

    def serve(self, requests, max_batch_seqs=0, hbm_fraction=0.5, realtime=True, keep_results=True, slots=0):
        """requests: list of (chars, offsets, distance, measure, arrival_s). Returns (per-request
        dicts with admitted_s, done_s, n_out, batch, status; per-request Result or None)."""
        keep = [(np.ascontiguousarray(c, dtype=np.uint8), np.ascontiguousarray(o, dtype=np.uint32))
                for c, o, *_ in requests]
        arr = (Request * max(1, len(requests)))()
        for i, ((c, o), (_, _, d, m, t)) in enumerate(zip(keep, requests)):
            arr[i] = Request(c.ctypes.data, o.ctypes.data, len(o) - 1, d, m, float(t))
        res = (RequestResult * max(1, len(requests)))()
        outs = [None] * len(requests)

        def cb(r, out_ptr, _user):
            if not keep_results:
                return
            o = out_ptr.contents
            if o.len <= 0:
                outs[r] = Result(np.zeros((0, 2), np.int32), np.zeros(0, np.int8), None)
                return
            pp = ctypes.cast(o.index_pairs, ctypes.POINTER(ctypes.c_int32))
            outs[r] = Result(np.ctypeslib.as_array(pp, shape=(o.len, 2)).copy(),
                             np.ctypeslib.as_array(o.pairwise_distances, shape=(o.len,)).copy(), None)

        ccb = REQUEST_CALLBACK(cb)
        opt = ServeOptions(max_batch_seqs, hbm_fraction, 1 if realtime else 0, slots)
        _check(self.lib.xtn_index_serve(self.h, arr, len(requests), ctypes.byref(opt), res, ccb, None))
        stats = [{k: getattr(res[i], k) for k, _ in RequestResult._fields_} for i in range(len(requests))]
        return stats, outs
