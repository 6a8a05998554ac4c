/*
 * xtn_b200 - C ABI of the B200 (sm_100a) symmetric-deletion neighbour search.
 *
 * This is the drop-in boundary for the hot path of XTNeighbor-streaming
 * (heartnetkung/XT-neighbor, xtneighbor_streaming/, abbreviated S/ below). The
 * reference exposes the path as one C++ function,
 *     void xtn_perform(XTNArgs, SeqArray*, SeqInfo*, void callback(XTNOutput))
 * (S/src/xtn.cu:267, declared S/src/xtn.h:124), called only by its CLI (S/src/cli.cu:267-271).
 * This header restates that interface with plain pointers and sizes so that any FFI
 * (ctypes, cgo, JNI, N-API) can bind it, and adds a reusable context, device-resident
 * entry points and status codes. All calls are synchronous with respect to the host
 * unless stated otherwise; a context may be used by one host thread at a time.
 */
#ifndef XTN_B200_H
#define XTN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Distance measures; same values as LEVENSHTEIN / HAMMING in S/src/xtn.h:12-14. */
#define XTN_LEVENSHTEIN 0
#define XTN_HAMMING 1

/* Return codes. 0..2 are the reference's ReturnCode {SUCCESS, ERROR, EXIT}
 * (S/src/xtn.h:93); the reference reports CUDA failures by printing and carrying on
 * (S/src/util.cu:5-11), this library returns one of the codes below instead. */
#define XTN_SUCCESS 0
#define XTN_ERROR 1
#define XTN_EXIT 2
#define XTN_ERR_CUDA 3      /* a CUDA call failed; xtn_last_error() has the text */
#define XTN_ERR_NOMEM 4     /* device or pinned-host allocation failed */
#define XTN_ERR_ARG 5       /* invalid argument (sizes, distance, measure, null pointers) */
#define XTN_ERR_NODEV 6     /* no usable CUDA device */
#define XTN_ERR_LIMIT 7     /* input exceeds a documented limit of this build */

/* Pair of sequence indexes; layout of Int2 (S/src/xtn.h:30-36). */
typedef struct xtn_int2 {
    int32_t x, y;
} xtn_int2;

/* Per-sequence information in overlap mode; layout of SeqInfo (S/src/xtn.h:41-45).
 * frequency: the row's count (non-zero int); repertoire: 0-based repertoire id, non-decreasing
 * over rows; original_index: the row's own index (the reference sets it, S/src/cli.cu:178-181). */
typedef struct xtn_seq_info {
    int32_t frequency, repertoire, original_index;
} xtn_seq_info;

/* Arguments; the fields of XTNArgs (S/src/xtn.h:50-60) that reach the algorithm.
 * The reference selects overlap mode with infoPath != NULL (S/src/xtn.cu:281); here a
 * non-null `info` argument does. */
typedef struct xtn_args {
    int32_t distance; /* >= 1 (S/src/cli.cu:53-57) */
    int32_t measure;  /* XTN_LEVENSHTEIN or XTN_HAMMING */
    int32_t verbose;  /* non-zero: print stage sizes and timings to stdout */
    int32_t info_len; /* overlap mode: number of repertoires (the -N value) */
} xtn_args;

/* One chunk of output; layout of XTNOutput (S/src/xtn.h:83-88).
 * NN mode: index_pairs[i] = (x, y), x < y, globally sorted by (x, y); pairwise_distances[i]
 * is the reference's `char` distance. Overlap mode: index_pairs[i] = (rep_x, rep_y) with
 * rep_x <= rep_y, sorted, and pairwise_frequencies[i] the summed count products (mod 2^64).
 * The arrays are owned by the library and valid only during the callback, as in the
 * reference (S/src/xtn.cu:458-459,479). */
typedef struct xtn_output {
    const xtn_int2* index_pairs;
    const int8_t* pairwise_distances;
    const uint64_t* pairwise_frequencies;
    int64_t len;
} xtn_output;

typedef void (*xtn_callback)(const xtn_output* output, void* user);

/* Opaque reusable state: device, streams and device buffers that grow on demand. */
typedef struct xtn_context xtn_context;

/* Counters and stage timings of the last run on a context. */
typedef struct xtn_stats {
    int64_t n_seqs;            /* sequences searched (unique sequences in overlap mode) */
    int64_t n_variants;        /* deletion variants generated */
    int64_t n_groups;          /* groups of equal variant hashes with >= 2 members */
    int64_t n_candidates;      /* candidate pairs emitted (with repeats and self-pairs) */
    int64_t n_unique;          /* distinct candidate pairs */
    int64_t n_out;             /* verified pairs (NN) or matrix entries (overlap) */
    int64_t n_verified_pairs;  /* verified sequence pairs (overlap mode) */
    int64_t n_launches;        /* kernel launches of the last run */
    int32_t id_bits;           /* bits used for a sequence id in packed records */
    int32_t n_rounds;          /* rounds the search ran in (contiguous ranges of first-level
                                  hash buckets sized to the memory budget; see memory_budget) */
    double ms_total;           /* device time of the last run, milliseconds */
    double ms_stage[8];        /* pack, gen, key sort, group, emit, pair sort, verify, output */
    int64_t n_fallback;        /* buckets grouped by sorting (too large for shared memory) */
} xtn_stats;

/* ------------------------------------------------------------------ reference interface */

/* xtn_perform: the whole search on host buffers; replaces S/src/xtn.cu:267-509.
 * seqs/offsets: CSR store of n_seqs sequences (what SeqArray holds after parsing,
 *   S/src/codec.cu:168-243): sequence i is seqs[offsets[i] .. offsets[i+1]), residues in
 *   'A'..'Y' minus B,J,O,U,X, length 1..500.
 * info: NULL for nearest-neighbour mode; in overlap mode one entry per row (row order).
 * callback is called one or more times with consecutive chunks of the sorted output.
 * Uses a library-owned context on device 0. Returns XTN_SUCCESS or an error code. */
int xtn_perform(const xtn_args* args, const char* seqs, const uint32_t* offsets, int32_t n_seqs,
                const xtn_seq_info* info, xtn_callback callback, void* user);

/* ------------------------------------------------------------------ context API */

int xtn_context_create(int device, xtn_context** out);
void xtn_context_destroy(xtn_context* ctx);

/* xtn_perform on an explicit context. */
int xtn_context_perform(xtn_context* ctx, const xtn_args* args, const char* seqs, const uint32_t* offsets,
                        int32_t n_seqs, const xtn_seq_info* info, xtn_callback callback, void* user);

/* Nearest-neighbour search on inputs already in device memory (d_seqs, d_offsets as in
 * xtn_perform). The result stays on the device; *n_out receives its length. Read it with
 * xtn_context_fetch or xtn_context_result_device. The offsets are checked on the device
 * before any kernel uses a length: a sequence outside 1..500 residues returns XTN_ERR_ARG
 * (the same check as xtn_perform's; the device-resident overlap and index entry points below
 * make it too). */
int xtn_context_nn_device(xtn_context* ctx, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                          int32_t n_seqs, int64_t* n_out);

/* Overlap mode on inputs already in device memory: d_info holds one xtn_seq_info per row
 * (row order) and args->info_len is the number of repertoires. The result (repertoire pairs
 * with their sums) stays on the device; *n_out receives its length. Read it with
 * xtn_context_fetch. Replaces the device-side part of xtn_perform's overlap mode
 * (xtneighbor_streaming/src/xtn.cu:267-509 with a non-null SeqInfo). */
int xtn_context_overlap_device(xtn_context* ctx, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                               int32_t n_seqs, const xtn_seq_info* d_info, int64_t* n_out);

/* Copies up to `cap` entries of the last result to host memory (either pointer may be NULL). */
int xtn_context_fetch(xtn_context* ctx, xtn_int2* pairs, int8_t* distances, uint64_t* frequencies, int64_t cap);

/* Device pointers of the last result (valid until the next run on the context). */
int xtn_context_result_device(xtn_context* ctx, const xtn_int2** d_pairs, const int8_t** d_distances, int64_t* n_out);

/* Shard exchange (multi-GPU search, options "shard_count" / "shard_index"). The reference runs
 * on one GPU and has no counterpart; these two calls are what a rank adds around its shard's
 * search.
 * xtn_context_result_keys writes the last nearest-neighbour result (sorted by (x, y)) to d_keys
 * (device memory, at least n_out entries) as one 64-bit key per pair,
 *   x << (b + 8) | y << 8 | (uint8_t)distance,   b = the smallest b >= 1 with 2^b >= n_seqs,
 * and range_starts[k] (host, n_ranges + 1 entries) = the first key whose x >= ceil(k n / K),
 * K = n_ranges, range_starts[K] = n_out: keys [range_starts[k], range_starts[k+1]) belong to
 * rank k's id range. xtn_context_merge_keys takes the keys a rank received (device memory, any
 * order, duplicates allowed), sorts them, drops repeats and leaves the pairs as the context's
 * result (xtn_context_fetch, *n_out entries): the ranks' results in rank order are the whole
 * search's output. */
int xtn_context_result_keys(xtn_context* ctx, int32_t n_seqs, uint64_t* d_keys, int64_t capacity, int32_t n_ranges,
                            int64_t* range_starts);
int xtn_context_merge_keys(xtn_context* ctx, int32_t n_seqs, const uint64_t* d_keys, int64_t count, int64_t* n_out);

/* Sharded search with a record exchange (the reference has no counterpart): every rank holds
 * the whole input and generates only the deletion variants of its own sequences
 * [rank n / K, (rank + 1) n / K).
 * xtn_shard_generate (rank `rank` of n_ranks): checks the lengths, packs all sequences (every
 * rank derives the same first-level shape from the whole search), generates and partitions its
 * own sequences' variant records into the search's first-level buckets. *n_buckets receives the
 * bucket count, bucket_counts[0..min(cap, n_buckets)) the records per bucket, *d_records /
 * *n_records the partitioned records in device memory (held by the context, valid until its
 * next call; bucket b's records follow bucket b - 1's). Needs distance <= 2 and the default
 * options key_tables = 1 and stage_chunk = 4096.
 * xtn_shard_search: d_records holds the n_pieces pieces a rank received for the b_n buckets it
 * owns (a contiguous range of the search's buckets), one after another; piece p holds
 * piece_counts[p * b_n + k] records of the rank's k-th bucket, in bucket order. The pieces are
 * gathered into contiguous buckets, split, grouped, de-duplicated, sorted and verified; the
 * verified pairs become the context's result (*n_out of them), to be exchanged by owner with
 * xtn_context_result_keys / xtn_context_merge_keys. */
int xtn_shard_generate(xtn_context* ctx, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                       int32_t n_seqs, int32_t rank, int32_t n_ranks, uint64_t* bucket_counts, int32_t cap,
                       int32_t* n_buckets, const uint64_t** d_records, int64_t* n_records);
int xtn_shard_search(xtn_context* ctx, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                     int32_t n_seqs, const uint64_t* d_records, const uint64_t* piece_counts, int32_t n_pieces,
                     int32_t b_n, int64_t* n_out);

/* The CUDA stream the context launches on (as a cudaStream_t cast to void*). */
void* xtn_context_stream(xtn_context* ctx);

int xtn_context_stats(const xtn_context* ctx, xtn_stats* out);

/* Per-kernel device time. With profiling on, every kernel launch of a run is bracketed by
 * CUDA events on the context stream; xtn_context_kernel_times then reports, per kernel
 * name, the summed duration (ms) and launch count of the last run. Returns the number of
 * distinct kernels (entries written: at most cap). */
int xtn_context_set_profiling(xtn_context* ctx, int on);
int xtn_context_kernel_times(const xtn_context* ctx, const char** names, double* ms, int64_t* launches, int cap);
/* Restricts profiling to the launches of one kernel name (as xtn_context_kernel_times reports
 * it), so that a timed run carries one pair of events per launch of that kernel only; NULL or
 * "" brackets every launch again. */
int xtn_context_profile_only(xtn_context* ctx, const char* name);

/* Tuning and engine options of a context (0 on success, XTN_ERR_ARG for an unknown name or
 * a value out of range):
 *   "engine"          0 = hash-bucket grouping in shared memory (default),
 *                     1 = full radix sort of the variant records (the plain comparison form)
 *   "bucket_bits_max" 1..14: upper bound on log2(number of first-level buckets) (default 10;
 *                     the search takes 512 buckets, or 1024 when they would exceed 1.5M
 *                     records). With the key tables (d <= 2) the stage shape's fan-out also
 *                     bounds it (10 for stage_chunk 4096, 9 for 2048); the direct scatter
 *                     (d > 2, key_tables = 0) takes up to 14
 *   "group_cap"       2..4096: largest bucket grouped in shared memory; larger ones are split
 *                     by further hash bits, and what still does not fit is grouped by sorting
 *                     (default 4096). At 2048 or below the grouping kernel takes its small
 *                     shape (256 threads and about 37 KB of shared memory: six CTAs per SM
 *                     instead of three)
 *   "scatter_ctas_per_sm" 0..4: first-level tiles per SM (default 0: as many CTAs as fit)
 *   "stage_chunk"     2048 | 4096 | 8192: records per shared-memory chunk of the first-level
 *                     scatter (default 4096: two CTAs of 512 threads per SM; 2048: four of 256;
 *                     8192: one of 1024, longer runs per bucket)
 *   "split_chunk"     2048 | 4096: the same for the split of large buckets; 8192: the one-pass
 *                     split (split_slotted) on 8192-record chunks, one CTA of 1024 threads per
 *                     SM (the two-pass split then takes 4096); 0 (default): 8192 for the
 *                     one-pass split when the first-level buckets average 2^20 records or
 *                     more, else 4096
 *   "split_fill"      25..95 (default 87): a first-level bucket larger than group_cap is split
 *                     into ceil(size / (group_cap * split_fill / 100)) sub-buckets (at most
 *                     1024) by ranges of the records' top hash bits, so the sub-buckets hold about
 *                     that share of the grouping capacity
 *   "split_slotted"   1 = the split runs in one pass: each sub-bucket gets a fixed slot of
 *                     group_cap records and every chunk reserves its runs there with one atomic
 *                     per sub-bucket (no histogram pass); a first-level bucket whose sub-bucket
 *                     outgrows its slot goes whole to the sort-based fallback (default);
 *                     0 = the two-pass split (a histogram pass merged across a cluster, then
 *                     exact placement)
 *   "split_slices"    1 | 8: CTAs per split bucket (default 8: one thread-block cluster whose
 *                     CTAs take slices of the bucket and merge their histograms through
 *                     distributed shared memory)
 *   "flat_gen"        1 = a search that keeps every record at once (one round, not sharded,
 *                     d <= 2, key tables, stage_chunk 4096) builds the first level in two
 *                     passes (default): every variant record generated in sequence order,
 *                     stored straight from the generating threads, with the per-tile bucket
 *                     histograms (in place of the count pass), then moved into its first-level
 *                     bucket by a streaming staged partition of 8192-record chunks; 0 = the
 *                     one-pass scatter that generates and partitions each chunk of 4096 (always
 *                     used in rounds and shards)
 *   "group_persistent" 1 = when there are many buckets to group (more than 8 per SM), the
 *                     grouping kernel runs as persistent CTAs that take bucket descriptors from
 *                     a queue on the device (default), 0 = one CTA per bucket
 *   "group_tma"       1 = load each bucket into shared memory with one TMA bulk copy
 *                     (default), 0 = with plain 16-byte loads from every thread
 *   "key_tables"      1 = for d <= 2, hash variants from per-sequence tables (default),
 *                     0 = hash each variant key directly (same hash values, slower)
 *   "onesweep"        1 = radix sorts of up to 2^24 keys (candidate pairs, fallback buckets)
 *                     by single-sweep passes with decoupled look-back (default; larger sorts
 *                     keep the classic passes), 0 = classic passes for every sort (per-tile
 *                     counts, a scan, a scatter)
 *   "pair_dedup"      1 = candidate pairs go through a hash set in HBM before the pair sort, so
 *                     only distinct pairs are sorted and verified (default; used from 2^15
 *                     candidates and for n <= 2^24), 0 = every candidate is sorted,
 *                     2 = as 1 with the table always sized from the previous search's share
 *                     of distinct pairs (the sizing used above 256 MiB of table)
 *   "dedup_slots_log2" 0 = size the one-round hash set as "pair_dedup" says (default);
 *                     16..30 = its first table has 2^this slots (a table found too full is
 *                     still regrown)
 *   "memory_budget"   bytes of device memory a search may hold (default 0: 80% of the free
 *                     device memory plus what the context holds, read only when one round
 *                     would need more than half of the device). A search whose variant
 *                     records do not fit runs in rounds over contiguous ranges of first-level
 *                     hash buckets (bucket engine; xtn_stats.n_rounds); a budget that cannot
 *                     hold one bucket returns XTN_ERR_NOMEM. Replaces the reference's memory
 *                     model and lower-bound rounds (xtneighbor_streaming/src/xtn.cu:21-26,
 *                     64-157, 383-470)
 *   "max_round_records" >= 0: at most this many variant records per round (default 0: no
 *                     bound beyond the budget and 2^32 - 2^20)
 *   "round_overlap"   1 = in a multi-round search, a round's candidate-pair dedup runs on a
 *                     second stream while the next round generates (default), 0 = in turn on
 *                     one stream
 *   "graph"           1 = xtn_context_nn_device runs the batched/persistent form: the whole
 *                     search (one round) is captured once per input (device pointers, size,
 *                     distance, measure, shape options) into a CUDA graph whose kernels read
 *                     every data-dependent size on the device (grouping by persistent CTAs
 *                     that take bucket descriptors from a device-side queue), and each later
 *                     search on that input replays it with one synchronisation at the end.
 *                     Capacities come from the plain search that precedes the capture; a
 *                     replay that exceeds one (or meets a bucket too large for shared memory)
 *                     is redone by the plain form, which re-sizes the graph. The same holds
 *                     for xtn_context_overlap_device: the string merge, diagonal term, the
 *                     search over the unique strings, cross term and matrix compaction form one
 *                     graph (per input and repertoire count); a replay whose unique-string
 *                     count differs from the capture's is redone by the plain form. A graph is
 *                     also re-captured when a search through another entry point has
 *                     reallocated the context's buffers. 0 = the plain form (default): one
 *                     launch sequence per search that reads sizes back to the host between
 *                     its stages
 *   "shard_count"     1..1024 (default 1) and
 *   "shard_index"     0..shard_count-1 (default 0): the nearest-neighbour search covers only
 *                     shard shard_index of shard_count - the first-level hash buckets whose
 *                     first record lies in [k V / K, (k + 1) V / K) of the V variant records,
 *                     so every group of equal variants lies in exactly one shard - and returns
 *                     that shard's verified pairs (sorted, unique within the shard). One rank
 *                     per GPU runs one shard on the same (replicated) input; the ranks then
 *                     exchange their pairs by owner (xtn_context_result_keys) and each merges
 *                     what it receives (xtn_context_merge_keys). Bucket engine only; the
 *                     overlap mode and the graph form run unsharded
 *   "verify_per"      1 | 4 | 8: the verification variant - candidates each lane of a warp lists
 *                     before the warp verifies them (default 1: the candidates are distinct
 *                     after the hash set, so listing more per lane only lengthens the warps;
 *                     4 or 8 amortise the listing when sorted candidates repeat)
 *   "autotune"        1 = xtn_context_nn_device takes its shape (the options the autotuner
 *                     sets) from the context's cache for the input's class, and on a miss runs
 *                     the autotuner on the input first (see xtn_context_autotune); 0 = the
 *                     shape is what the options say (default)
 *   "wait_polls"      1..4194304: bound on the polls of one look-back wait in the single-pass
 *                     prefix sums (default 4194304); a wait that reaches it makes the call
 *                     return XTN_ERR_CUDA and the result is discarded
 *   "wait_fault_test" 1 = the next search's variant-offset prefix sum leaves its first tile's
 *                     status word unset, so the later tiles' bounded waits run out: the call
 *                     returns XTN_ERR_CUDA and the context stays usable (a test of the error
 *                     path; reset to 0 after that one search) */
int xtn_context_set_option(xtn_context* ctx, const char* name, int64_t value);

/* Autotuner: times the search on these device-resident inputs (the caller's data, so its length
 * distribution and duplicate structure) for each shape - the first-level form (two passes or
 * the one-pass scatter), first-level and split stage chunks and first-level bucket bits, then,
 * on the best of those, bulk-copy or plain loads in the grouping
 * kernel, the verification variants (verify_per 4 and 8) and the graph form - taking the best of
 * `repeats` runs after a warm-up, and leaves the fastest shape set on the context. The choice is
 * also remembered for the input's class (log2 of the sequence count, distance, measure, median
 * sequence length, share of sequences longer than the 18-residue key), which option "autotune"
 * uses. `report` (may be NULL) receives the choice, its time and the class. No counterpart in
 * the reference, which has fixed chunk sizes (xtneighbor_streaming/src/xtn.cu:21-26). */
int xtn_context_autotune(xtn_context* ctx, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                         int32_t n_seqs, int32_t repeats, char* report, int32_t report_cap);

/* ------------------------------------------------------------------ resident index and serving */

/* A resident deletion index: every deletion variant (at most max_distance <= 2 deletions) of
 * the first 18 residues of n_seqs reference sequences, hashed, tagged with its deletion count
 * and sorted in device memory, with a directory on the top hash bits. It has no counterpart
 * in the reference, which only runs whole offline searches (xtneighbor_streaming/src/xtn.cu:
 * 267-509); a query batch is answered exactly as that offline search would answer the
 * sequences (index rows 0..n_seqs-1 followed by the batch), restricted to the pairs with one
 * index row x and one batch row q: pairs (x, n_seqs + q) in (x, y) order with the reference
 * distance. Inputs as in xtn_perform. Owns a context (stream and scratch) on `device`. */
typedef struct xtn_index xtn_index;

typedef struct {
    int64_t n_seqs;
    int64_t n_records;      /* deletion variants held */
    int64_t bytes;          /* device memory held by the index */
    int32_t max_distance;
    int32_t directory_bits; /* log2 of the directory size */
    double ms_build;        /* device time of the build */
} xtn_index_info;

int xtn_index_create(int device, const char* seqs, const uint32_t* offsets, int32_t n_seqs, int32_t max_distance,
                     xtn_index** out);
/* The same from device-resident inputs (copied: the caller may free them afterwards). */
int xtn_index_create_device(int device, const char* d_seqs, const uint32_t* d_offsets, int32_t n_seqs,
                            int32_t max_distance, xtn_index** out);
void xtn_index_destroy(xtn_index* index);
int xtn_index_stats(const xtn_index* index, xtn_index_info* out);
/* The index's context: its stream, stats, kernel times and last query result
 * (xtn_context_fetch / xtn_context_result_device). */
xtn_context* xtn_index_context(xtn_index* index);

/* One query batch from host buffers; args->distance <= max_distance. The result reaches the
 * callback in chunks, as in xtn_perform. */
int xtn_index_query(xtn_index* index, const xtn_args* args, const char* seqs, const uint32_t* offsets,
                    int32_t n_queries, xtn_callback callback, void* user);
/* One query batch from device buffers; the result stays on the index's context. */
int xtn_index_query_device(xtn_index* index, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                           int32_t n_queries, int64_t* n_out);

/* Serving loop with continuous batching. Requests (host buffers) arrive at arrival_s seconds
 * after the call starts (realtime) or all at once. The loop runs `slots` batches at a time, each
 * slot on its own stream and host thread with its own query scratch (slot 0 uses the index's
 * context); the index itself is shared, read only. Whenever a slot is free it admits the ready
 * requests of the oldest one's (distance, measure) in arrival order while the batch fits the
 * slot's memory budget (hbm_fraction of the device memory free when the loop starts, split
 * over the slots, after buffers for the largest request are reserved in each slot; at most
 * max_batch_seqs sequences), runs them as one query batch, splits the answer by request and
 * hands each request its pairs (y = n_seqs + the request's own row) through the callback. So a
 * request that arrives while another slot runs a large batch starts at once, and their work
 * overlaps on the device. A request larger than the budget runs in pieces. A request's
 * answer does not depend on the batch it joins (each pair is found and verified from the
 * request's own sequences). Callbacks come from the loop's threads, one at a time.
 * results[i] receives the admission and completion times (seconds since the call started), the
 * batch, the pair count and the status of request i. */
typedef struct {
    const char* seqs;
    const uint32_t* offsets;
    int32_t n_seqs;
    int32_t distance;
    int32_t measure;
    double arrival_s;
} xtn_request;

typedef struct {
    double admitted_s;
    double done_s;
    int64_t n_out;
    int32_t batch;
    int32_t status;
} xtn_request_result;

typedef struct {
    int64_t max_batch_seqs; /* <= 0: 2^20 */
    double hbm_fraction;    /* of free device memory the batches may use; <= 0: 0.5 */
    int32_t realtime;       /* 1: honour arrival_s; 0: every request is ready at once */
    int32_t slots;          /* batches in flight at a time, 1..8; <= 0: 2 */
} xtn_serve_options;

typedef void (*xtn_request_callback)(int32_t request, const xtn_output* out, void* user);

int xtn_index_serve(xtn_index* index, const xtn_request* requests, int32_t n_requests,
                    const xtn_serve_options* options, xtn_request_result* results, xtn_request_callback callback,
                    void* user);

/* ------------------------------------------------------------------ search without allocation */

/* Nearest-neighbour search that allocates nothing. It has no counterpart in the reference.
 * Meant for callers that cannot allocate device memory while they run:
 *   - a host whose framework caching allocator already holds the device memory;
 *   - a latency-critical loop that cannot take the synchronisation of cudaMalloc/cudaFree;
 *   - a plugin host that forbids allocation on the call path.
 * The caller passes device pointers: the sequences (as in xtn_perform) and output buffers of
 * out_cap pairs and distances. The result is the same as xtn_context_nn_device's, written to
 * the caller's buffers, with its length in *n_out (a host pointer).
 *
 * Limits and behaviour:
 *   - Scratch comes from one fixed 32 MiB device array inside the library, held by every GPU
 *     that loads it until the process exits. The array is reserved when the library's device
 *     code is loaded on a device; with CUDA's lazy module loading that can be during this
 *     function's first call there, so a caller that must not see any allocation on its call
 *     path makes one warm-up call per device first.
 *   - The caller's offsets are checked on the device (1..500 residues per sequence); a bad
 *     length returns XTN_ERR_ARG naming the first bad sequence.
 *   - At most 4096 sequences. Inputs whose variants, groups or candidate pairs do not fit the
 *     array, or whose result exceeds out_cap, return XTN_ERR_LIMIT with a message. For an
 *     oversized result, *n_out holds the needed size.
 *   - Runs on `stream` (a cudaStream_t, NULL for the legacy default stream) on the current
 *     device, and returns after the stream has drained.
 *   - The first call on a device also resolves the array's device address.
 *   - Every call reuses the same array (the call resets what must start at zero), so calls that
 *     overlap on the GPU, from any thread or stream, race. */
int xtn_nn_search_static(const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets, int32_t n_seqs,
                         xtn_int2* d_out_pairs, int8_t* d_out_distances, int64_t out_cap, int64_t* n_out,
                         void* stream);

/* Text of the last error on the calling thread ("" if none). */
const char* xtn_last_error(void);

/* Library version string ("2.0.0" like the reference CLI, S/src/cli.cu:9, plus a build tag). */
const char* xtn_version(void);

#ifdef __cplusplus
}
#endif

#endif /* XTN_B200_H */
