// Hash-bucket grouping of deletion variants (the default key-grouping engine).
//
// The sort-based engine orders all V variant records by hash with a multi-pass radix sort
// (about 24 bytes of HBM traffic per record per 8-bit digit). Grouping only needs equal
// hashes to meet, not a global order, so this engine moves each 8-byte record through HBM a
// fixed small number of times. First level, when the search keeps every record at once:
//   gen      k_bucket_gen      every variant hashed from the key tables by balanced tasks
//                              and stored in sequence order, (hash & ~idmask) | id, with the
//                              per-tile histogram of the top b1 hash bits
//   offsets  k_bucket_colscan  per bucket: exclusive prefix over tiles, bucket totals
//   partition k_bucket_partition
//                              each tile's records, read back by bulk copies, through a staged
//                              partition into their first-level buckets (every global store
//                              part of a coalesced run, so L2 receives whole sectors)
// First level in rounds and shards (records of a bucket range only), or at d > 2:
//   count    k_bucket_count    per tile: histogram of the top b1 hash bits (not stored)
//   scatter  k_bucket_scatter_staged / k_bucket_scatter
//                              the variants again, up to 4096 at a time in shared memory,
//                              ranked within their bucket as they are made and written out as
//                              contiguous runs (or stored directly at d > 2)
// Then:
//   plan     k_bucket_plan     buckets that fit in shared memory go straight to grouping;
//                              larger ones are split by ranges of their next hash bits into
//                              sub-buckets of about split_fill % of the grouping capacity
//   split    k_bucket_split_slotted (+ k_split_slot_descs), or k_bucket_split_staged
//                              per oversized bucket, the staged partition into sub-buckets:
//                              in one pass into fixed slots with a cursor per sub-bucket, or in
//                              two (histograms merged across a cluster, exact placement)
//   group    k_bucket_group    one CTA per (sub-)bucket (persistent CTAs on a queue): TMA bulk
//                              copy into shared memory, a bitmap filter that drops records
//                              without a partner, a counting sort of the rest, runs of equal
//                              hashes, then every id pair of every run, spread evenly over the
//                              CTA's threads and written with coalesced stores
// Buckets that still exceed shared memory after the split (one variant shared by very many
// sequences) are grouped by the sort-based path instead, in batches.
#pragma once
#include <cstdint>

#include <cooperative_groups.h>

#include "xtn_common.cuh"

namespace xtn {

constexpr int kBucketThreads = 512;    // k_bucket_count and the direct scatter (d > 2)
constexpr int kPrivFan = 64;           // split fan-outs up to this use per-warp histograms
// First-level fan-out: a staged chunk of 2048..4096 records leaves runs of 4..8 records
// (32..64 bytes) per bucket; consecutive chunks of one CTA extend the same runs, so their
// boundary sectors complete in L2.
constexpr int kMaxFirstLevelBits = 10;  // default bound on the first-level bits (the large stage shape's fan-out)
constexpr int kMaxSplitBits = 10;
constexpr int kMaxSplitFan = 1 << kMaxSplitBits;  // sub-buckets of one split job, at most
// CTAs (one thread-block cluster) per split bucket (16, the non-portable cluster size, measured
// slower at 10M: 8.24 against 7.40 ms)
constexpr int kSplitSlices = 8;

// Shape of a staged partition: threads per CTA, records per chunk, largest fan-out.
template <int THREADS, int CHUNK, int FAN>
struct StageCfg {
    static constexpr int kThreads = THREADS;
    static constexpr int kChunk = CHUNK;
    static constexpr int kFan = FAN;
    static constexpr int kFanPer = FAN / THREADS;
    static constexpr int kPer = CHUNK / THREADS;
    static_assert(FAN % THREADS == 0 && CHUNK % THREADS == 0 && CHUNK <= 65536, "stage shape");
};
using StageLarge = StageCfg<512, 4096, 1024>;  // ~110 KB of shared memory: two CTAs per SM
using StageSmall = StageCfg<256, 2048, 512>;   // ~55 KB: four CTAs per SM (first level, b1 <= 9)
// ~210 KB: one CTA of 1024 threads per SM (first level only): with 1024 first-level buckets a
// chunk of 8192 records leaves runs of about eight records (64 bytes) per bucket instead of four
using StageHuge = StageCfg<1024, 8192, 1024>;
using SplitSmall = StageCfg<256, 2048, 1024>;  // ~60 KB: three CTAs per SM
// Shape of a grouping CTA: records it holds in shared memory, threads, hash bits of the
// "seen" / "seen twice" bitmaps, hash bits of the candidates' counting sort, and minimum CTAs per
// SM. The large shape (~65 KB of shared memory, three CTAs per SM) holds buckets of up to 4096
// records; the small one (~37 KB, six CTAs of 256 threads per SM) holds up to 2048, which the
// split produces when group_cap <= 2048.
template <int CAP, int THREADS, int BITMAP_LOG, int DIGIT_BITS, int MIN_CTAS>
struct GroupCfg {
    static constexpr int kCap = CAP;
    static constexpr int kThreads = THREADS;
    static constexpr int kBitmapLog = BITMAP_LOG;
    static constexpr int kBitmapBits = 1 << BITMAP_LOG;
    static constexpr int kBitmapWords = kBitmapBits / 32;
    static constexpr int kDigitBits = DIGIT_BITS;
    static constexpr int kDigits = 1 << DIGIT_BITS;
    static constexpr int kMinCtas = MIN_CTAS;
    static_assert(kDigits % THREADS == 0 && CAP < 65536, "group shape");
};
// (One digit per thread, 512 / 256 digits, measured slower on the 10M workload: 10.03 against
// 9.90 ms, as more candidates share a digit.)
using GroupLarge = GroupCfg<4096, 512, 16, 11, 3>;
using GroupSmall = GroupCfg<2048, 256, 15, 10, 6>;
// (Half the bitmap and digits at the large cap, 2^15 bits and 1024 digits, measured slower:
// 9.32 against 8.99 ms at 10M, 0.80 against 0.70 ms at 1M.)
constexpr int kGroupThreads = GroupLarge::kThreads;
constexpr int kGroupCap = GroupLarge::kCap;        // largest bucket grouped in shared memory
constexpr int kGroupSmallCap = GroupSmall::kCap;   // group_cap at or below this: the small shape
// Runs of >= 2 equal hashes one grouping CTA lists (a full bucket could hold up to CAP / 2;
// buckets with more than this go to the sort-based fallback).
constexpr int kMaxRuns = 1024;

// Descriptor of one bucket (or sub-bucket) handed to the grouping kernel.
struct BucketDesc {
    uint64_t start;   // first record
    uint32_t size;    // records
    uint32_t src;     // 0: records in buffer A, 1: in buffer B
};

// Split job: bucket `start,size` (buffer A) is divided into `nsub` sub-buckets (buffer B) by
// ranges of the records' top hash bits (split_sub).
struct SplitJob {
    uint64_t start;
    uint32_t size;
    uint32_t nsub;
    uint32_t sub0;   // the job's first sub-bucket among all jobs' (slotted split)
    uint32_t pad;
};

// Sub-bucket of record x among nsub: the top 32 hash bits scaled to [0, nsub), so that any
// count of near-equal sub-buckets can be made (not only powers of two); equal records land in
// the same one.
__device__ __forceinline__ uint32_t split_sub(uint64_t x, uint32_t nsub) { return __umulhi((uint32_t)(x >> 32), nsub); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Exclusive scan of one value per thread across a block of THREADS threads.
template <typename T, int THREADS>
__device__ __forceinline__ T block_scan_ex(T v, T* total, T* warp_sums) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < THREADS / 32 ? warp_sums[lane] : T(0);
        T winc = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T t = __shfl_up_sync(0xffffffffu, winc, o);
            if (lane >= o) winc += t;
        }
        if (lane < THREADS / 32) warp_sums[lane] = winc - w;
        if (lane == THREADS / 32 - 1) warp_sums[THREADS / 32] = winc;
    }
    __syncthreads();
    T r = inc - v + warp_sums[warp];
    *total = warp_sums[THREADS / 32];
    __syncthreads();
    return r;
}

// ------------------------------------------------------------------ count
// Per-tile histogram of the variants' first-level buckets; d <= 2 hashes come from the key
// tables when given.
__global__ void __launch_bounds__(kBucketThreads) k_bucket_count(const u128* __restrict__ keys,
                                                                 const uint8_t* __restrict__ klen,
                                                                 const uint64_t* __restrict__ runinfo,
                                                                 const uint64_t* __restrict__ tab, int n, int tile, int d,
                                                                 int b1, uint32_t* __restrict__ counts) {
    extern __shared__ uint32_t s_hist[];
    const int nb = 1 << b1;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    const int base = blockIdx.x * tile;
    const int end = min(n, base + tile);
    const int shift = 64 - b1;
    if (tab && d <= 2)
        for (int i = base + threadIdx.x; i < end; i += blockDim.x)
            for_each_hash(tab + (size_t)i * kTabLen, klen[i], runinfo[i], d,
                          [&](uint64_t h) { atomicAdd(&s_hist[h >> shift], 1u); });
    else
        for (int i = base + threadIdx.x; i < end; i += blockDim.x)
            for_each_variant(keys[i], klen[i], d, [&](u128 k) { atomicAdd(&s_hist[key_hash(k) >> shift], 1u); });
    __syncthreads();
    uint32_t* out = counts + (size_t)blockIdx.x * nb;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) out[i] = s_hist[i];
}

// counts/offsets are tile-major [tile][bucket]; offsets become the exclusive prefix over tiles.
// Per bucket, the exclusive prefix of its tile counts and its total. A block takes 32 buckets
// (one per lane, so that every row read is one 128-byte line) and its warps split the tiles:
// each warp sums its share, then writes its prefixes from the warps before it. (One thread per
// bucket over all tiles, two blocks at 512 buckets, took 0.2 ms at 10M sequences.)
constexpr int kColscanWarps = 32;

__global__ void __launch_bounds__(kColscanWarps * 32) k_bucket_colscan(const uint32_t* __restrict__ counts, int ntiles,
                                                                      int nb, uint32_t* __restrict__ offsets,
                                                                      uint32_t* __restrict__ totals) {
    __shared__ uint32_t s_part[kColscanWarps][33];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int b = blockIdx.x * 32 + lane;
    const int per = (ntiles + kColscanWarps - 1) / kColscanWarps;
    const int t0 = min(ntiles, w * per), t1 = min(ntiles, t0 + per);
    uint32_t sum = 0;
    if (b < nb)
        for (int t = t0; t < t1; t++) sum += counts[(size_t)t * nb + b];
    s_part[w][lane] = sum;
    __syncthreads();
    uint32_t run = 0;
    for (int k = 0; k < w; k++) run += s_part[k][lane];
    if (b >= nb) return;
    for (int t = t0; t < t1; t++) {
        const uint32_t c = counts[(size_t)t * nb + b];
        offsets[(size_t)t * nb + b] = run;
        run += c;
    }
    if (w == kColscanWarps - 1) totals[b] = run;
}

// Counter words shared by the plan, split and grouping kernels (unsigned int counters[16]).
constexpr int kCntDesc = 0;      // descriptors listed for grouping
constexpr int kCntJobs = 1;      // split jobs
constexpr int kCntSub = 2;       // sub-buckets the split jobs produce
constexpr int kCntFallback = 3;  // buckets grouped by sorting instead
constexpr int kCntWaitFail = 5;  // split and partition CTAs whose chunk copy did not complete in time
constexpr int kCntDropped = 6;   // appends refused because a list was full (must stay 0)

// ------------------------------------------------------------------ staged partition
template <class C>
struct StageSmem {
    uint64_t rec[C::kChunk + 2]; // records of the chunk, in arrival order (+ bulk-copy alignment)
    uint64_t sorted[C::kChunk];  // the same records grouped by bucket
    uint16_t sbkt[C::kChunk];    // bucket of sorted[i]
    uint32_t cnt[C::kFan];
    uint32_t lstart[C::kFan];
    uint32_t gcur[C::kFan];      // next global position of each bucket for this CTA
    uint32_t warp_sums[C::kThreads / 32 + 1];
    uint32_t wait_failed;
    unsigned long long mbar;     // completion barrier of the chunk bulk copies (split)
};

// Resident CTAs per SM that a stage shape's shared memory allows (228 KB per SM, 1 KB
// reserved per CTA).
template <class C>
constexpr int stage_ctas_per_sm() {
    return (int)((228u * 1024u) / (sizeof(StageSmem<C>) + 1024u));
}

// Staged partition of a split chunk: the chunk's records are r[0..m), the bucket of r[p] is
// r[p] >> shift; each bucket's records are appended at gcur[bucket] as contiguous runs written by
// consecutive threads. after_rank() runs once every thread is done reading r.
// `strip` > 0 (first level from records in sequence order): a record x = hash field | id
// carries its bucket in its top `strip` bits. They are dropped on the way out and the field
// shifted up by `strip`, as the one-pass scatter's records are; the `strip` bits that opens
// above the id take a multiplicative hash of the whole field, so that the low field bits, which
// the grouping's bitmap filter indexes, vary within a bucket (equal fields still give equal
// records; the field keeps 64 - idbits - strip bits of the hash, against 64 - idbits for the
// one-pass scatter, so a bucket sees a few more hash collisions, which verification removes).
__device__ __forceinline__ uint64_t strip_bucket(uint64_t x, int strip, int idbits) {
    const uint64_t idmask = (1ull << idbits) - 1ull;
    const uint64_t f = x & ~idmask;
    const uint64_t mix = (f * 0x9E3779B97F4A7C15ull) >> (64 - strip);
    return (f << strip) | (mix << idbits) | (x & idmask);
}

template <class C, class Bkt, class Hook>
__device__ __forceinline__ void split_partition(StageSmem<C>& S, int nb, uint32_t m, const uint64_t* r, Bkt&& bkt,
                                                uint64_t* __restrict__ dst, Hook&& after_rank, int strip = 0,
                                                int idbits = 0) {
    constexpr int kStageThreads = C::kThreads, kFanPer = C::kFanPer;
    for (int b = threadIdx.x; b < nb; b += kStageThreads) S.cnt[b] = 0;
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < m; p += kStageThreads) atomicAdd(&S.cnt[bkt(r[p])], 1u);
    __syncthreads();
    {
        uint32_t tot, loc[kFanPer], sum = 0;
        const int b0 = threadIdx.x * kFanPer;
#pragma unroll
        for (int k = 0; k < kFanPer; k++) {
            loc[k] = sum;
            sum += (b0 + k < nb) ? S.cnt[b0 + k] : 0u;
        }
        const uint32_t ex = block_scan_ex<uint32_t, kStageThreads>(sum, &tot, S.warp_sums);
#pragma unroll
        for (int k = 0; k < kFanPer; k++)
            if (b0 + k < nb) {
                S.lstart[b0 + k] = ex + loc[k];
                S.cnt[b0 + k] = ex + loc[k];
            }
    }
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < m; p += kStageThreads) {
        const uint64_t x = r[p];
        const uint32_t b = bkt(x);
        const uint32_t q = atomicAdd(&S.cnt[b], 1u);
        S.sorted[q] = x;
        S.sbkt[q] = (uint16_t)b;
    }
    __syncthreads();
    after_rank();
    for (uint32_t q = threadIdx.x; q < m; q += kStageThreads) {
        const uint16_t b = S.sbkt[q];
        const uint64_t x = S.sorted[q];
        dst[S.gcur[b] + (q - S.lstart[b])] = strip ? strip_bucket(x, strip, idbits) : x;
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nb; b += kStageThreads) S.gcur[b] += S.cnt[b] - S.lstart[b];
    __syncthreads();
}

// The staged partition with one shared-memory atomic per record: the counting atomic returns the
// record's rank within its bucket, kept in a register (bucket << 16 | rank; a chunk holds at most
// 2^16 records and a stage at most 2^16 buckets) until the scan has placed the buckets, so that
// no second ranking pass reads the chunk again. KEEP: the records stay in registers as well, the
// chunk buffer is free once every thread has read it, and after_read() (the next chunk's bulk
// copy) runs before the scan instead of after the ranking. (k_bucket_partition: 4.90 against
// 5.10 ms at 10M.)
template <class C, bool KEEP, class Bkt, class Hook>
__device__ __forceinline__ void split_partition_ranked(StageSmem<C>& S, int nb, uint32_t m, const uint64_t* r,
                                                       Bkt&& bkt, uint64_t* __restrict__ dst, Hook&& after_read,
                                                       int strip, int idbits) {
    constexpr int T = C::kThreads, kFanPer = C::kFanPer, kPer = C::kPer;
    static_assert(C::kChunk <= 65536 && C::kFan <= 65536, "rank word");
    for (int b = threadIdx.x; b < nb; b += T) S.cnt[b] = 0;
    __syncthreads();
    uint32_t rk[kPer];
    uint64_t xs[KEEP ? kPer : 1];
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        const uint32_t p = threadIdx.x + (uint32_t)k * T;
        rk[k] = ~0u;
        if (p < m) {
            const uint64_t x = r[p];
            if (KEEP) xs[k] = x;
            const uint32_t b = bkt(x);
            rk[k] = (b << 16) | atomicAdd(&S.cnt[b], 1u);
        }
    }
    __syncthreads();
    if (KEEP) after_read();
    {
        uint32_t tot, loc[kFanPer], sum = 0;
        const int b0 = threadIdx.x * kFanPer;
#pragma unroll
        for (int k = 0; k < kFanPer; k++) {
            loc[k] = sum;
            sum += (b0 + k < nb) ? S.cnt[b0 + k] : 0u;
        }
        const uint32_t ex = block_scan_ex<uint32_t, T>(sum, &tot, S.warp_sums);
#pragma unroll
        for (int k = 0; k < kFanPer; k++)
            if (b0 + k < nb) S.lstart[b0 + k] = ex + loc[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        if (rk[k] == ~0u) continue;
        const uint32_t b = rk[k] >> 16;
        const uint32_t q = S.lstart[b] + (rk[k] & 0xffffu);
        S.sorted[q] = KEEP ? xs[k] : r[threadIdx.x + (uint32_t)k * T];
        S.sbkt[q] = (uint16_t)b;
    }
    __syncthreads();
    if (!KEEP) after_read();
    for (uint32_t q = threadIdx.x; q < m; q += T) {
        const uint16_t b = S.sbkt[q];
        const uint64_t x = S.sorted[q];
        dst[S.gcur[b] + (q - S.lstart[b])] = strip ? strip_bucket(x, strip, idbits) : x;
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nb; b += T) S.gcur[b] += S.cnt[b];
    __syncthreads();
}

constexpr uint32_t kWaitLimit = 1u << 26;  // bound on mbarrier polls

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(mbar), "r"(phase)
        : "memory");
    return ok != 0;
}

// One bulk copy of `bytes` (a multiple of 16) from 16-byte aligned global memory into shared
// memory, completing on `mbar` (issued by one thread).
__device__ __forceinline__ void bulk_load(uint32_t dst_smem, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     dst_smem),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}

// Tasks per sequence for the first-level generation at d = 2: 2 * ceil(runs / 2) balanced
// tasks (task_items). (At d = 1 each sequence is one task and needs no map.)
__global__ void k_task_counts(const uint64_t* __restrict__ runinfo, int n, uint32_t* __restrict__ tcnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t R = (uint32_t)popc32((uint32_t)runinfo[i]);
    tcnt[i] = 2u * ((R + 1u) >> 1);
}

// Task -> sequence map of the staged scatter: the k_task_counts tasks of sequence i occupy
// task_seq[toff[i] .. toff[i+1]).
// The CTA's sequences write their task ids into shared memory (at most kKeyLen tasks each), then
// the CTA stores its contiguous task range with consecutive threads on consecutive words.
constexpr int kTaskSeqThreads = 256;

__global__ void __launch_bounds__(kTaskSeqThreads) k_task_seq(const uint64_t* __restrict__ toff, int n,
                                                              uint32_t* __restrict__ task_seq) {
    __shared__ uint32_t s_ids[kTaskSeqThreads * kKeyLen];
    const int i0 = blockIdx.x * kTaskSeqThreads;
    const int i = i0 + threadIdx.x;
    const int i1 = min(n, i0 + kTaskSeqThreads);
    const uint64_t base = toff[i0];
    if (i < n)
        for (uint64_t g = toff[i], e = toff[i + 1]; g < e; g++) s_ids[g - base] = (uint32_t)i;
    __syncthreads();
    const uint32_t cnt = (uint32_t)(toff[i1] - base);
    for (uint32_t k = threadIdx.x; k < cnt; k += kTaskSeqThreads) task_seq[base + k] = s_ids[k];
}

constexpr int kMaxVariantsD2 = 1 + kKeyLen + kKeyLen * (kKeyLen - 1) / 2;  // 172: all runs of length 1
constexpr int kScatterChunksPerRound = 1024;

template <class C>
struct ScatterSmem {
    uint64_t rec[C::kChunk];     // records of the chunk, at their sequence's slots
    uint64_t sorted[C::kChunk];  // the same records grouped by bucket
    uint32_t br[C::kChunk];      // bucket << 16 | rank of rec[i] among the chunk's records of its bucket
    uint32_t dst[C::kChunk];     // global position of sorted[i]
    uint32_t cnt[C::kFan];       // records of each bucket in the chunk
    uint32_t lstart[C::kFan];    // first slot of each bucket in `sorted`
    uint32_t gcur[C::kFan];      // next global position of each bucket for this CTA
    uint32_t cstart[kScatterChunksPerRound + 1];
    uint32_t warp_sums[C::kThreads / 32 + 1];
    uint32_t m_in;               // records of the chunk inside the round's bucket range
};

template <class SM>
constexpr int ctas_per_sm_for() {
    return (int)((228u * 1024u) / (sizeof(SM) + 1024u));
}

// Chunks of a tile of sequences [t0, t1) for the staged first-level kernels: chunk k holds the
// sequences whose first variant lies in [k * span, (k + 1) * span) from voff[r0], with
// span = CHUNK - 172 (a key has at most 172 variants at d <= 2), so that no chunk overflows and
// none is empty. Fills cstart[0..nch] (at most kScatterChunksPerRound chunks per call, from r0);
// returns nch. The caller synchronises before reading cstart.
template <int T, int CHUNK>
__device__ __forceinline__ int chunk_starts(const uint64_t* __restrict__ voff, int r0, int t1, uint32_t* cstart) {
    constexpr uint64_t kSpan = (uint64_t)(CHUNK - kMaxVariantsD2);
    const uint64_t base = voff[r0];
    const uint64_t last = (voff[t1 - 1] - base) / kSpan;
    const int nch = last + 1 < (uint64_t)kScatterChunksPerRound ? (int)(last + 1) : kScatterChunksPerRound;
    for (int s = r0 + threadIdx.x; s < t1; s += T) {
        const uint64_t k = (voff[s] - base) / kSpan;
        if (k > (uint64_t)nch) break;
        if (s == r0 || (voff[s - 1] - base) / kSpan != k) cstart[k] = (uint32_t)s;
    }
    if (threadIdx.x == 0 && (uint64_t)nch == last + 1) cstart[nch] = (uint32_t)t1;
    return nch;
}

// The variant hashes of the chunk of sequences [s0, s1) (d <= 2, from the key tables): the
// chunk's generation tasks are spread over the CTA's T threads and put(pos, hash, seq) is
// called once per variant, pos = its slot in the chunk (voff[seq] - voff[s0] + the variant's
// index). At d = 2 the tasks are k_task_counts' balanced halves of run pairs and task_seq maps a
// task to its sequence; at d = 1 (task_seq null) a task is a whole sequence: its table row is
// loaded into registers at once and the key and single deletions are emitted by an unrolled
// loop.
template <int T, class Put>
__device__ __forceinline__ void chunk_hashes(const uint8_t* __restrict__ klen, const uint64_t* __restrict__ runinfo,
                                             const uint64_t* __restrict__ tab, const uint64_t* __restrict__ voff,
                                             const uint64_t* __restrict__ toff, const uint32_t* __restrict__ task_seq,
                                             int s0, int s1, int d, Put&& put) {
    const uint64_t vbase = voff[s0];
    const uint64_t tb = task_seq ? toff[s0] : (uint64_t)s0;
    const uint32_t nt = (uint32_t)((task_seq ? toff[s1] : (uint64_t)s1) - tb);
    for (uint32_t tau = threadIdx.x; tau < nt; tau += T) {
        const uint64_t g = tb + tau;
        const int i = task_seq ? (int)task_seq[g] : (int)g;
        const int t = task_seq ? (int)(g - toff[i]) : 0;
        const uint32_t vb = (uint32_t)(voff[i] - vbase);
        auto emit = [&](int v, uint64_t h) { put(vb + (uint32_t)v, h, i); };
        const uint64_t* row = tab + (size_t)i * kTabLen;
        if (d >= 2) {
            for_each_task_hash(row, klen[i], runinfo[i], d, t, emit);
        } else {
            // the key, then the single deletion of each run: r G[p] + r^-1 P_L
            uint64_t G[kKeyLen];
#pragma unroll
            for (int q = 0; q < kKeyLen; q++) G[q] = row[kTabG + q];
            const uint64_t PL = row[kTabKey];
            const uint32_t rs = (uint32_t)runinfo[i];
            emit(0, hash_fin(PL));
            const uint64_t single = kPolyRI * PL;
            int v = 1;
#pragma unroll
            for (int q = 0; q < kKeyLen; q++)
                if ((rs >> q) & 1u) emit(v++, hash_fin(kPolyR * G[q] + single));
        }
    }
}

// First-level scatter for d <= 2. The CTA's tile of sequences is cut into chunks of at most
// C::kChunk variants by a rule every thread can apply alone: chunk k holds the sequences whose
// first variant lies in [k * span, (k + 1) * span) from the tile's first variant, with
// span = C::kChunk - 172 (a key has at most 172 variants at d <= 2), so no chunk overflows
// and none is empty. For each chunk:
//   1. the chunk's generation tasks hash their variants from the key tables (one load and one
//      add per variant), write each record at its sequence's slot and take its rank within
//      its bucket with one shared-memory atomic. At d = 2 the tasks are k_task_counts'
//      balanced halves of run pairs and task_seq maps a task to its sequence; at d = 1
//      (task_seq null) a task is a whole sequence: its table row is loaded into registers
//      at once and the key and single deletions are emitted by an unrolled loop;
//   2. an exclusive scan of the bucket counts, a rank-ordered copy into `sorted`, and
//      coalesced writes of each bucket's run at the CTA's cursor (gcur).
// runinfo[i] is key_run_info of sequence i, tab its key_table; voff and toff are exclusive
// scans of the variant and task counts (toff = sequence index at d = 1).
// Rounds: only the records of buckets [b_lo, b_lo + b_n) are kept, at their global position
// minus `round_base` (the global position of bucket b_lo's first record); the others are
// generated and dropped (b_lo = 0, b_n = 2^b1, round_base = 0: every record, one round).
template <class C>
__global__ void __launch_bounds__(C::kThreads, ctas_per_sm_for<ScatterSmem<C>>()) k_bucket_scatter_staged(
    const uint8_t* __restrict__ klen, const uint64_t* __restrict__ runinfo, const uint64_t* __restrict__ tab,
    const uint64_t* __restrict__ voff, const uint64_t* __restrict__ toff, const uint32_t* __restrict__ task_seq, int n,
    int tile, int d, int b1, int idbits, const uint32_t* __restrict__ offsets, const uint64_t* __restrict__ bstart,
    uint32_t b_lo, uint32_t b_n, uint64_t round_base, uint64_t* __restrict__ recs,
    const unsigned int* __restrict__ abort) {
    constexpr int T = C::kThreads, kFanPer = C::kFanPer;
    if (abort && *abort) return;  // graph form: the records would not fit their buffer
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ScatterSmem<C>& S = *reinterpret_cast<ScatterSmem<C>*>(smem_raw);
    const int nb = 1 << b1;
    const uint32_t* off = offsets + (size_t)blockIdx.x * nb;
    for (int b = threadIdx.x; b < nb; b += T) {
        S.gcur[b] = (uint32_t)(bstart[b] - round_base) + off[b];  // used for buckets of the round only
        S.cnt[b] = 0;
    }
    const int t0 = blockIdx.x * tile;
    const int t1 = min(n, t0 + tile);
    const int shift = 64 - b1;
    const uint64_t hi_mask = ~((1ull << idbits) - 1ull);
    for (int r0 = t0; r0 < t1;) {
        // chunk starts of this round (at most kScatterChunksPerRound chunks)
        const int nch = chunk_starts<T, C::kChunk>(voff, r0, t1, S.cstart);
        __syncthreads();
        for (int c = 0; c < nch; c++) {
            const int s0 = (int)S.cstart[c], s1 = (int)S.cstart[c + 1];
            const uint32_t m = (uint32_t)(voff[s1] - voff[s0]);
            chunk_hashes<T>(klen, runinfo, tab, voff, toff, task_seq, s0, s1, d, [&](uint32_t pos, uint64_t h, int i) {
                const uint32_t b = (uint32_t)(h >> shift);
                if (b - b_lo >= b_n) {  // another round's bucket
                    S.br[pos] = 0xffffffffu;
                    return;
                }
                S.br[pos] = (b << 16) | atomicAdd(&S.cnt[b], 1u);
                S.rec[pos] = ((h << b1) & hi_mask) | (uint64_t)i;
            });
            __syncthreads();
            {
                uint32_t tot, loc[kFanPer], sum = 0;
                const int b0 = threadIdx.x * kFanPer;
#pragma unroll
                for (int k = 0; k < kFanPer; k++) {
                    loc[k] = sum;
                    sum += (b0 + k < nb) ? S.cnt[b0 + k] : 0u;
                }
                const uint32_t ex = block_scan_ex<uint32_t, T>(sum, &tot, S.warp_sums);
#pragma unroll
                for (int k = 0; k < kFanPer; k++)
                    if (b0 + k < nb) S.lstart[b0 + k] = ex + loc[k];
                if (threadIdx.x == 0) S.m_in = tot;
            }
            __syncthreads();
            for (uint32_t p = threadIdx.x; p < m; p += T) {
                const uint32_t br = S.br[p], b = br >> 16, r = br & 0xffffu;
                if (br == 0xffffffffu) continue;
                const uint32_t q = S.lstart[b] + r;
                S.sorted[q] = S.rec[p];
                S.dst[q] = S.gcur[b] + r;
            }
            __syncthreads();
            const uint32_t m_in = S.m_in;
            for (uint32_t q = threadIdx.x; q < m_in; q += T) recs[S.dst[q]] = S.sorted[q];
            __syncthreads();
            for (int b = threadIdx.x; b < nb; b += T) {
                S.gcur[b] += S.cnt[b];
                S.cnt[b] = 0;
            }
            __syncthreads();
        }
        r0 = (int)S.cstart[nch];
        __syncthreads();
    }
}

// ------------------------------------------------------------------ generate, then partition
// The first level in two passes (searches that keep every record at once, d <= 2 with key
// tables): k_bucket_gen writes every variant record in sequence order, (hash & ~idmask) | id,
// and the per-tile histogram of the top b1 hash bits (the count pass's output, so that pass is
// not run); k_bucket_partition then moves each tile's records, read back by bulk copies, through
// the staged partition into their first-level buckets. Generation has no chunks, ranking or
// barriers, and the partition is a streaming pass with known offsets; the one-pass scatter
// interleaves both inside each chunk of 4096 records.
//
// k_bucket_gen: the tile's generation tasks are spread over the CTA at once and every variant
// is stored straight to its slot; a lane's consecutive variants fill whole sectors, which L2
// merges before they reach DRAM (two CTAs of 512 threads per SM at 64 registers; a bound of
// three CTAs measured slower: 6.46 against 5.55 ms at 10M, one thread per sequence instead of
// the balanced tasks 12.7 ms, and whole run-pair tasks instead of halves 7.2 ms. Ordering the
// tasks by item count within groups of 32 sequences, so that a warp's loops have equal length
// (95% instead of 83% of its issue slots busy), measured slower too: 7.1 ms, as a warp's lanes
// then read 32 sequences' table rows and write into 32 sequences' records per instruction
// instead of two or three; 14.2 ms within groups of 256; the bucket shift as a compile-time
// constant for 512 buckets: 5.58 ms, no faster). abort (graph
// form, may be null): the records would not fit. The tiles cover sequences [seq0, n), whose
// records start at record rec0 = voff[seq0] (a shard of a search: flat holds only those).
template <int THREADS, int MIN_CTAS>
__global__ void __launch_bounds__(THREADS, MIN_CTAS) k_bucket_gen(
    const uint8_t* __restrict__ klen, const uint64_t* __restrict__ runinfo, const uint64_t* __restrict__ tab,
    const uint64_t* __restrict__ voff, const uint64_t* __restrict__ toff, const uint32_t* __restrict__ task_seq, int n,
    int tile, int d, int b1, int idbits, uint64_t* __restrict__ flat, uint32_t* __restrict__ counts,
    const unsigned int* __restrict__ abort, int seq0, uint64_t rec0) {
    extern __shared__ uint32_t s_hist[];
    if (abort && *abort) return;
    const int nb = 1 << b1;
    for (int b = threadIdx.x; b < nb; b += THREADS) s_hist[b] = 0;
    __syncthreads();
    const int t0 = (int)min((int64_t)n, (int64_t)seq0 + (int64_t)blockIdx.x * tile);
    const int t1 = min(n, t0 + tile);
    const int shift = 64 - b1;
    const uint64_t hi_mask = ~((1ull << idbits) - 1ull);
    if (t0 < t1) {
        uint64_t* out = flat + (voff[t0] - rec0);
        chunk_hashes<THREADS>(klen, runinfo, tab, voff, toff, task_seq, t0, t1, d,
                                    [&](uint32_t pos, uint64_t h, int i) {
                                        atomicAdd(&s_hist[(uint32_t)(h >> shift)], 1u);
                                        out[pos] = (h & hi_mask) | (uint64_t)i;
                                    });
    }
    __syncthreads();
    uint32_t* dst = counts + (size_t)blockIdx.x * nb;
    for (int b = threadIdx.x; b < nb; b += THREADS) dst[b] = s_hist[b];
}

// k_bucket_partition: tile t's records, flat[voff[t * tile] .. voff[min(n, (t + 1) * tile)]),
// (tiles from sequence seq0 on, flat starting at record rec0 = voff[seq0], as k_bucket_gen)
// through the staged partition into their first-level buckets in `recs`: bucket b's records of
// tile t start at bstart[b] + offsets[t][b]; the top b1 bits are dropped on the way
// (strip_bucket). Chunk c reaches shared memory by one bulk copy, issued as soon as chunk c - 1
// is ranked; counters[kCntWaitFail] counts CTAs whose bounded wait for a copy ran out. The
// 8192-record stage shape (one CTA of 1024 threads per SM) leaves runs of about eight records
// per bucket and chunk at 1024 first-level buckets.
template <class C>
__global__ void __launch_bounds__(C::kThreads) k_bucket_partition(
    const uint64_t* __restrict__ flat, const uint64_t* __restrict__ voff, int n, int tile, int b1, int idbits,
    const uint32_t* __restrict__ offsets, const uint64_t* __restrict__ bstart, uint64_t* __restrict__ recs,
    unsigned int* __restrict__ counters, const unsigned int* __restrict__ abort, int seq0, uint64_t rec0) {
    constexpr int T = C::kThreads;
    if (abort && *abort) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StageSmem<C>& S = *reinterpret_cast<StageSmem<C>*>(smem_raw);
    const int nb = 1 << b1;
    // (tiles past the last sequence are empty)
    const int t0 = (int)min((int64_t)n, (int64_t)seq0 + (int64_t)blockIdx.x * tile);
    const int t1 = min(n, t0 + tile);
    const uint32_t* off = offsets + (size_t)blockIdx.x * nb;
    for (int b = threadIdx.x; b < nb; b += T) S.gcur[b] = (uint32_t)bstart[b] + off[b];
    const uint64_t r0 = voff[t0];
    const uint32_t size = (uint32_t)(voff[t1] - r0);
    const uint64_t* src = flat + (r0 - rec0);
    const uint32_t mbar = smem_u32(&S.mbar);
    auto issue = [&](uint32_t c0) {
        const uint32_t m = min((uint32_t)C::kChunk, size - c0);
        const uint64_t* a = src + c0;
        const uint32_t lead = (uint32_t)(((uintptr_t)a & 15u) >> 3);
        bulk_load(smem_u32(&S.rec[0]), a - lead, ((lead + m) * 8u + 15u) & ~15u, mbar);
    };
    if (threadIdx.x == 0) {
        S.wait_failed = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (size > 0) issue(0);
    }
    __syncthreads();
    uint32_t parity = 0;
    for (uint32_t c0 = 0; c0 < size; c0 += C::kChunk, parity ^= 1u) {
        const uint32_t m = min((uint32_t)C::kChunk, size - c0);
        const uint32_t lead = (uint32_t)(((uintptr_t)(src + c0) & 15u) >> 3);
        if (threadIdx.x == 0) {
            uint32_t polls = 0;
            while (!mbar_try_wait(mbar, parity)) {
                if (++polls > kWaitLimit) {
                    S.wait_failed = 1;
                    break;
                }
                __nanosleep(32);
            }
        }
        __syncthreads();
        if (S.wait_failed) {
            // one more bounded wait for the copy to land before the shared memory is released
            if (threadIdx.x == 0) {
                uint32_t polls = 0;
                while (!mbar_try_wait(mbar, parity) && ++polls < kWaitLimit) __nanosleep(64);
                atomicAdd(&counters[kCntWaitFail], 1u);
            }
            __syncthreads();
            return;
        }
        const int shift = 64 - b1;
        split_partition_ranked<C, true>(S, nb, m, S.rec + lead, [shift](uint64_t x) { return (uint32_t)(x >> shift); },
                                        recs, [&] {
                                            if (threadIdx.x == 0 && c0 + C::kChunk < size) issue(c0 + C::kChunk);
                                        }, b1, idbits);
    }
}

// First-level scatter for any d: one thread per sequence, smem cursors, direct stores. Rounds
// as in k_bucket_scatter_staged: buckets [b_lo, b_lo + b_n) only, positions minus `round_base`.
__global__ void __launch_bounds__(kBucketThreads) k_bucket_scatter(const u128* __restrict__ keys,
                                                                   const uint8_t* __restrict__ klen, int n, int tile, int d,
                                                                   int b1, int idbits, const uint32_t* __restrict__ offsets,
                                                                   const uint64_t* __restrict__ bstart, uint32_t b_lo,
                                                                   uint32_t b_n, uint64_t round_base,
                                                                   uint64_t* __restrict__ recs,
                                                                   const unsigned int* __restrict__ abort) {
    if (abort && *abort) return;
    extern __shared__ uint32_t s_cur[];
    const int nb = 1 << b1;
    const uint32_t* off = offsets + (size_t)blockIdx.x * nb;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s_cur[i] = (uint32_t)(bstart[i] - round_base) + off[i];
    __syncthreads();
    const int base = blockIdx.x * tile;
    const int end = min(n, base + tile);
    const int shift = 64 - b1;
    const uint64_t hi_mask = ~((1ull << idbits) - 1ull);
    for (int i = base + threadIdx.x; i < end; i += blockDim.x) {
        const uint64_t id = (uint64_t)i;
        for_each_variant(keys[i], klen[i], d, [&](u128 k) {
            uint64_t h = key_hash(k);
            const uint32_t b = (uint32_t)(h >> shift);
            if (b - b_lo >= b_n) return;
            uint32_t pos = atomicAdd(&s_cur[b], 1u);
            recs[pos] = ((h << b1) & hi_mask) | id;
        });
    }
}


// Appends v to list[0..cap) at counters[which]; an append past the capacity is counted in
// counters[kCntDropped] instead (the host then reports an error: the capacities are bounds
// that the plan's arithmetic guarantees, so this never happens with consistent inputs).
template <class T>
__device__ __forceinline__ void bounded_append(T* __restrict__ list, uint32_t cap, unsigned int* __restrict__ counters,
                                               int which, const T& v) {
    const unsigned k = atomicAdd(&counters[which], 1u);
    if (k < cap) list[k] = v;
    else atomicAdd(&counters[kCntDropped], 1u);
}

// Sorts buckets into "group directly" descriptors and split jobs.
// bstart points at the round's first bucket; `base` is that bucket's global start, so the
// descriptors hold positions in the round's record buffer.
// abort (graph form, may be null): when set, nothing is listed, so the split and grouping that
// follow have no work.
__global__ void k_bucket_plan(const uint64_t* __restrict__ bstart, int nb, uint64_t base, uint32_t group_cap,
                              uint32_t split_fill, BucketDesc* __restrict__ desc, uint32_t desc_cap,
                              SplitJob* __restrict__ jobs, unsigned int* __restrict__ counters,
                              const unsigned int* __restrict__ abort) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb || (abort && *abort)) return;
    uint64_t s = bstart[b] - base, e = bstart[b + 1] - base;
    uint32_t size = (uint32_t)(e - s);
    if (size < 2) return;
    if (size <= group_cap) {
        bounded_append(desc, desc_cap, counters, kCntDesc, BucketDesc{s, size, 0});
    } else {
        // sub-buckets of about split_fill % of the shared-memory capacity (hash buckets are
        // near-uniform, so the largest stays below the capacity)
        const uint64_t target = max(1u, (uint32_t)((uint64_t)group_cap * split_fill / 100));
        const uint64_t want = (size + target - 1) / target;
        const uint32_t nsub = want < 2 ? 2u : want > (uint64_t)kMaxSplitFan ? (uint32_t)kMaxSplitFan : (uint32_t)want;
        const uint32_t sub0 = atomicAdd(&counters[kCntSub], nsub);
        bounded_append(jobs, (uint32_t)nb, counters, kCntJobs, SplitJob{s, size, nsub, sub0, 0});
    }
}

// Split of the oversized first-level buckets. Each job (bucket) is handled by a cluster of
// kSlices CTAs, each taking a contiguous slice of the bucket's records:
//   1. each CTA histograms its slice by sub-bucket (split_sub: ranges of the top hash bits);
//   2. after a cluster barrier, each CTA reads every slice's histogram from its peers' shared
//      memory (distributed shared memory, plain loads) and derives the sub-bucket totals, their
//      starts and its own offset inside each sub-bucket; rank 0 lists the sub-buckets (those
//      that fit for grouping, larger ones for the fallback); a second barrier ends the remote
//      reads;
//   3. each CTA streams its slice chunk by chunk (bulk copy, the next chunk in flight during the
//      write-out) through the staged partition into buffer B at the bucket's range.
// With kSlices CTAs per bucket, few buckets are in flight at a time, so the second read of a
// slice comes from L2 rather than DRAM. counters[5] counts CTAs whose chunk copy did not
// complete within the wait bound (their output is incomplete; the host reports an error).
template <class C, int kSlices>
__global__ void __cluster_dims__(kSlices, 1, 1) __launch_bounds__(C::kThreads, stage_ctas_per_sm<C>())
    k_bucket_split_staged(const SplitJob* __restrict__ jobs, const uint64_t* __restrict__ in,
                          uint64_t* __restrict__ out, uint32_t group_cap, BucketDesc* __restrict__ desc,
                          BucketDesc* __restrict__ fallback, uint32_t desc_cap, unsigned int* __restrict__ counters) {
    constexpr int kStageThreads = C::kThreads, kStageChunk = C::kChunk, kFanPer = C::kFanPer;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StageSmem<C>& S = *reinterpret_cast<StageSmem<C>*>(smem_raw);
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    if (blockIdx.x / kSlices >= min(counters[kCntJobs], (unsigned)(gridDim.x / kSlices))) return;  // no such job
    const SplitJob job = jobs[blockIdx.x / kSlices];
    const uint32_t nsub = job.nsub;
    const bool priv = nsub <= (uint32_t)kPrivFan;
    const uint32_t s_lo = (uint32_t)((uint64_t)job.size * rank / kSlices);
    const uint32_t s_hi = (uint32_t)((uint64_t)job.size * (rank + 1) / kSlices);
    const uint32_t size = s_hi - s_lo;
    const uint64_t* src = in + job.start + s_lo;
    // Chunk c of the slice reaches S.rec by one bulk copy from the 16-byte boundary at or below
    // its first record (the record buffers carry 16 bytes of padding), completing on S.mbar
    // with parity c & 1. The copy of chunk c + 1 is issued as soon as chunk c's records are
    // ranked, so it overlaps chunk c's write-out.
    const uint32_t mbar = smem_u32(&S.mbar);
    auto issue = [&](uint32_t c0) {
        const uint32_t m = min((uint32_t)kStageChunk, size - c0);
        const uint64_t* a = src + c0;
        const uint32_t lead = (uint32_t)(((uintptr_t)a & 15u) >> 3);
        bulk_load(smem_u32(&S.rec[0]), a - lead, ((lead + m) * 8u + 15u) & ~15u, mbar);
    };
    if (threadIdx.x == 0) {
        S.wait_failed = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (size > 0) issue(0);
    }
    // 1. slice histogram into S.lstart (per-warp copies in `sorted`, unused until the first
    //    chunk, for small fan-outs)
    uint32_t* hist = priv ? reinterpret_cast<uint32_t*>(S.sorted) + (threadIdx.x >> 5) * kPrivFan : S.lstart;
    for (int i = threadIdx.x; i < (priv ? kPrivFan * (kStageThreads / 32) : (int)nsub); i += kStageThreads)
        (priv ? reinterpret_cast<uint32_t*>(S.sorted) : S.lstart)[i] = 0;
    __syncthreads();
    {
        // 16-byte loads, four in flight per thread (the slice is 8-byte aligned: peel one)
        const uint32_t lead = size > 0 ? (uint32_t)(((uintptr_t)src & 15u) >> 3) : 0u;
        if (lead && threadIdx.x == 0) atomicAdd(&hist[split_sub(src[0], nsub)], 1u);
        const uint32_t nv = (size - lead) >> 1;
        const uint4* v = reinterpret_cast<const uint4*>(src + lead);
        uint32_t i = threadIdx.x;
        for (; i + 3 * kStageThreads < nv; i += 4 * kStageThreads) {
            const uint4 w[4] = {__ldg(v + i), __ldg(v + i + kStageThreads), __ldg(v + i + 2 * kStageThreads),
                                __ldg(v + i + 3 * kStageThreads)};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                atomicAdd(&hist[__umulhi(w[k].y, nsub)], 1u);  // (the top 32 bits of each record)
                atomicAdd(&hist[__umulhi(w[k].w, nsub)], 1u);
            }
        }
        for (; i < nv; i += kStageThreads) {
            const uint4 a = __ldg(v + i);
            atomicAdd(&hist[__umulhi(a.y, nsub)], 1u);
            atomicAdd(&hist[__umulhi(a.w, nsub)], 1u);
        }
        if (threadIdx.x == 0 && ((size - lead) & 1u)) atomicAdd(&hist[split_sub(src[size - 1], nsub)], 1u);
    }
    __syncthreads();
    if (priv) {
        for (int b = threadIdx.x; b < (int)nsub; b += kStageThreads) {
            uint32_t t = 0;
            for (int w = 0; w < kStageThreads / 32; w++) t += reinterpret_cast<uint32_t*>(S.sorted)[w * kPrivFan + b];
            S.lstart[b] = t;
        }
    }
    cluster.sync();
    // 2. sub-bucket totals, starts and this slice's offsets from every slice's histogram
    {
        uint32_t tot_b[kFanPer], mine_b[kFanPer], loc[kFanPer], sum = 0;
        const int b0 = threadIdx.x * kFanPer;
#pragma unroll
        for (int k = 0; k < kFanPer; k++) {
            tot_b[k] = mine_b[k] = 0;
            if (b0 + k < (int)nsub)
                for (int r = 0; r < kSlices; r++) {
                    const uint32_t c = cluster.map_shared_rank(S.lstart, r)[b0 + k];
                    tot_b[k] += c;
                    if (r < rank) mine_b[k] += c;
                }
            loc[k] = sum;
            sum += tot_b[k];
        }
        uint32_t tot;
        const uint32_t ex = block_scan_ex<uint32_t, kStageThreads>(sum, &tot, S.warp_sums);
#pragma unroll
        for (int k = 0; k < kFanPer; k++) {
            const int b = b0 + k;
            if (b >= (int)nsub) continue;
            const uint32_t st = ex + loc[k];
            S.gcur[b] = (uint32_t)job.start + st + mine_b[k];
            if (rank == 0 && tot_b[k] >= 2) {
                BucketDesc bd{job.start + st, tot_b[k], 1};
                if (tot_b[k] <= group_cap) bounded_append(desc, desc_cap, counters, kCntDesc, bd);
                else bounded_append(fallback, desc_cap, counters, kCntFallback, bd);
            }
        }
    }
    cluster.sync();  // no remote reads after this point: S.lstart is free again
    // 3. the slice through the staged partition
    uint32_t parity = 0;
    for (uint32_t c0 = 0; c0 < size; c0 += kStageChunk, parity ^= 1u) {
        const uint32_t m = min((uint32_t)kStageChunk, size - c0);
        const uint32_t lead = (uint32_t)(((uintptr_t)(src + c0) & 15u) >> 3);
        if (threadIdx.x == 0) {
            uint32_t polls = 0;
            while (!mbar_try_wait(mbar, parity)) {
                if (++polls > kWaitLimit) {
                    S.wait_failed = 1;
                    break;
                }
                __nanosleep(32);
            }
        }
        __syncthreads();
        if (S.wait_failed) {
            // one more bounded wait for the copy to land before the shared memory is released
            if (threadIdx.x == 0) {
                uint32_t polls = 0;
                while (!mbar_try_wait(mbar, parity) && ++polls < kWaitLimit) __nanosleep(64);
                atomicAdd(&counters[kCntWaitFail], 1u);
            }
            __syncthreads();
            return;
        }
        split_partition(S, (int)nsub, m, S.rec + lead, [nsub](uint64_t x) { return split_sub(x, nsub); }, out, [&] {
            if (threadIdx.x == 0 && c0 + kStageChunk < size) issue(c0 + kStageChunk);
        });
    }
}

// ------------------------------------------------------------------ shard exchange
// A run of records copied from `src` to `dst` (received pieces gathered into contiguous
// first-level buckets).
struct GatherRun {
    uint64_t src, dst;
    uint64_t size;
};

__global__ void k_gather_runs(const GatherRun* __restrict__ runs, const uint64_t* __restrict__ src,
                              uint64_t* __restrict__ dst) {
    const GatherRun r = runs[blockIdx.x];
    for (uint64_t i = threadIdx.x; i < r.size; i += blockDim.x) dst[r.dst + i] = src[r.src + i];
}

// ------------------------------------------------------------------ slotted split
// The split in one pass over the records: every sub-bucket gets a slot of `slot` records (the
// grouping capacity) in buffer B at (job.sub0 + sub) * slot, and each chunk of a slice, after
// its staged ranking, reserves its runs with one global atomic per sub-bucket on that
// sub-bucket's cursor and writes them there. No histogram pass, no cluster: kSlices CTAs take
// slices of a job independently. Records past a slot's end are not written but counted, so a
// cursor above `slot` marks a sub-bucket too large for shared memory; k_split_slot_descs then
// lists the job's whole first-level bucket for the sort-based fallback instead (the other
// sub-buckets' pairs it also finds again are removed with the other repeats).
template <class C, int kSlices>
__global__ void __launch_bounds__(C::kThreads, stage_ctas_per_sm<C>())
    k_bucket_split_slotted(const SplitJob* __restrict__ jobs, const uint64_t* __restrict__ in,
                           uint64_t* __restrict__ out, uint32_t slot, unsigned int* __restrict__ cursors,
                           unsigned int* __restrict__ counters, const unsigned int* __restrict__ abort) {
    constexpr int T = C::kThreads, kChunk = C::kChunk, kFanPer = C::kFanPer;
    // the 8192-record stage (one CTA of 1024 threads per SM, 64 registers a thread) keeps a
    // chunk's records in registers; the 4096-record one (two CTAs per SM) reads them twice
    constexpr bool kKeep = C::kChunk >= 8192;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StageSmem<C>& S = *reinterpret_cast<StageSmem<C>*>(smem_raw);
    if (abort && *abort) return;
    if (blockIdx.x / kSlices >= min(counters[kCntJobs], (unsigned)(gridDim.x / kSlices))) return;  // no such job
    const SplitJob job = jobs[blockIdx.x / kSlices];
    const int rank = (int)(blockIdx.x % kSlices);
    const uint32_t nsub = job.nsub;
    const uint32_t s_lo = (uint32_t)((uint64_t)job.size * rank / kSlices);
    const uint32_t s_hi = (uint32_t)((uint64_t)job.size * (rank + 1) / kSlices);
    const uint32_t size = s_hi - s_lo;
    const uint64_t* src = in + job.start + s_lo;
    uint64_t* dst = out + (uint64_t)job.sub0 * slot;
    unsigned int* cur = cursors + job.sub0;
    const uint32_t mbar = smem_u32(&S.mbar);
    auto issue = [&](uint32_t c0) {
        const uint32_t m = min((uint32_t)kChunk, size - c0);
        const uint64_t* a = src + c0;
        const uint32_t lead = (uint32_t)(((uintptr_t)a & 15u) >> 3);
        bulk_load(smem_u32(&S.rec[0]), a - lead, ((lead + m) * 8u + 15u) & ~15u, mbar);
    };
    if (threadIdx.x == 0) {
        S.wait_failed = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (size > 0) issue(0);
    }
    __syncthreads();
    uint32_t parity = 0;
    for (uint32_t c0 = 0; c0 < size; c0 += kChunk, parity ^= 1u) {
        const uint32_t m = min((uint32_t)kChunk, size - c0);
        const uint32_t lead = (uint32_t)(((uintptr_t)(src + c0) & 15u) >> 3);
        if (threadIdx.x == 0) {
            uint32_t polls = 0;
            while (!mbar_try_wait(mbar, parity)) {
                if (++polls > kWaitLimit) {
                    S.wait_failed = 1;
                    break;
                }
                __nanosleep(32);
            }
        }
        __syncthreads();
        if (S.wait_failed) {
            if (threadIdx.x == 0) {
                uint32_t polls = 0;
                while (!mbar_try_wait(mbar, parity) && ++polls < kWaitLimit) __nanosleep(64);
                atomicAdd(&counters[kCntWaitFail], 1u);
            }
            __syncthreads();
            return;
        }
        const uint64_t* r = S.rec + lead;
        for (uint32_t b = threadIdx.x; b < nsub; b += T) S.cnt[b] = 0;
        __syncthreads();
        if constexpr (kKeep) {
            // records and their ranks stay in registers (split_partition_ranked): one shared
            // atomic per record, and the next chunk's copy starts once the chunk is read
            uint32_t rk[C::kPer];
            uint64_t xs[C::kPer];
#pragma unroll
            for (int k = 0; k < C::kPer; k++) {
                const uint32_t p = threadIdx.x + (uint32_t)k * T;
                rk[k] = ~0u;
                xs[k] = 0;
                if (p < m) {
                    xs[k] = r[p];
                    const uint32_t b = split_sub(xs[k], nsub);
                    rk[k] = (b << 16) | atomicAdd(&S.cnt[b], 1u);
                }
            }
            __syncthreads();
            if (threadIdx.x == 0 && c0 + kChunk < size) issue(c0 + kChunk);
            {
                uint32_t tot, loc[kFanPer], cnt[kFanPer], sum = 0;
                const int b0 = threadIdx.x * kFanPer;
#pragma unroll
                for (int k = 0; k < kFanPer; k++) {
                    loc[k] = sum;
                    cnt[k] = (b0 + k < (int)nsub) ? S.cnt[b0 + k] : 0u;
                    sum += cnt[k];
                }
                const uint32_t ex = block_scan_ex<uint32_t, T>(sum, &tot, S.warp_sums);
#pragma unroll
                for (int k = 0; k < kFanPer; k++)
                    if (cnt[k]) {
                        S.lstart[b0 + k] = ex + loc[k];
                        S.gcur[b0 + k] = atomicAdd(&cur[b0 + k], cnt[k]);  // this chunk's runs in the slot
                    }
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < C::kPer; k++) {
                if (rk[k] == ~0u) continue;
                const uint32_t b = rk[k] >> 16;
                const uint32_t q = S.lstart[b] + (rk[k] & 0xffffu);
                S.sorted[q] = xs[k];
                S.sbkt[q] = (uint16_t)b;
            }
            __syncthreads();
        } else {
            for (uint32_t p = threadIdx.x; p < m; p += T) atomicAdd(&S.cnt[split_sub(r[p], nsub)], 1u);
            __syncthreads();
            {
                uint32_t tot, loc[kFanPer], cnt[kFanPer], sum = 0;
                const int b0 = threadIdx.x * kFanPer;
#pragma unroll
                for (int k = 0; k < kFanPer; k++) {
                    loc[k] = sum;
                    cnt[k] = (b0 + k < (int)nsub) ? S.cnt[b0 + k] : 0u;
                    sum += cnt[k];
                }
                const uint32_t ex = block_scan_ex<uint32_t, T>(sum, &tot, S.warp_sums);
#pragma unroll
                for (int k = 0; k < kFanPer; k++)
                    if (cnt[k]) {
                        S.lstart[b0 + k] = ex + loc[k];
                        S.cnt[b0 + k] = ex + loc[k];
                        S.gcur[b0 + k] = atomicAdd(&cur[b0 + k], cnt[k]);  // this chunk's runs in the slot
                    }
            }
            __syncthreads();
            // (the ranks kept in registers from the counting pass, as split_partition_ranked does,
            // measured slower here: 5.53 against 5.44 ms at 10M)
            for (uint32_t p = threadIdx.x; p < m; p += T) {
                const uint64_t x = r[p];
                const uint32_t b = split_sub(x, nsub);
                const uint32_t q = atomicAdd(&S.cnt[b], 1u);
                S.sorted[q] = x;
                S.sbkt[q] = (uint16_t)b;
            }
            __syncthreads();
            if (threadIdx.x == 0 && c0 + kChunk < size) issue(c0 + kChunk);
        }
        for (uint32_t q = threadIdx.x; q < m; q += T) {
            const uint16_t b = S.sbkt[q];
            const uint32_t pos = S.gcur[b] + (q - S.lstart[b]);
            if (pos < slot) dst[(uint64_t)b * slot + pos] = S.sorted[q];
        }
        __syncthreads();
    }
}

// Descriptors of the slotted split, one CTA per job: the sub-buckets of two or more records
// (slot positions, buffer B), or, when any sub-bucket outgrew its slot, the job's whole
// first-level bucket (buffer A) for the sort-based fallback.
__global__ void k_split_slot_descs(const SplitJob* __restrict__ jobs, const unsigned int* __restrict__ cursors,
                                   uint32_t slot, BucketDesc* __restrict__ desc, BucketDesc* __restrict__ fallback,
                                   uint32_t desc_cap, unsigned int* __restrict__ counters,
                                   const unsigned int* __restrict__ abort) {
    if (abort && *abort) return;
    if (blockIdx.x >= counters[kCntJobs]) return;
    const SplitJob job = jobs[blockIdx.x];
    const unsigned int* cur = cursors + job.sub0;
    int over = 0;
    for (uint32_t b = threadIdx.x; b < job.nsub; b += blockDim.x) over |= cur[b] > slot;
    if (__syncthreads_or(over)) {
        if (threadIdx.x == 0) bounded_append(fallback, desc_cap, counters, kCntFallback, BucketDesc{job.start, job.size, 0});
        return;
    }
    for (uint32_t b = threadIdx.x; b < job.nsub; b += blockDim.x) {
        const uint32_t c = cur[b];
        if (c >= 2) bounded_append(desc, desc_cap, counters, kCntDesc, BucketDesc{(uint64_t)(job.sub0 + b) * slot, c, 1});
    }
}

// ------------------------------------------------------------------ group
// Shared-memory layout of k_bucket_group (about 65 KB: three CTAs per SM). The two bitmaps
// are only needed until the candidates are known; the grouping arrays reuse their space.
template <class G>
struct GroupSmem {
    uint64_t rec[G::kCap + 2];  // bucket records (+ alignment slack)
    union {
        struct {
            uint32_t seen[G::kBitmapWords];   // hash bit seen once
            uint32_t twice[G::kBitmapWords];  // hash bit seen at least twice
        } bm;
        struct {
            uint16_t perm[G::kCap];    // candidate record indexes grouped by digit
            uint32_t runs[kMaxRuns];   // contiguous << 31 | size << 16 | head slot, per run of >= 2
            uint32_t poff[kMaxRuns];   // first pair index of each run
        } gr;
    } u;
    uint16_t cand[G::kCap];     // records whose bitmap bit was hit at least twice
    uint32_t cnt[G::kDigits];   // digit counts -> digit ends
    uint32_t warp_sums[G::kThreads / 32 + 1];
    unsigned long long warp_sums64[G::kThreads / 32 + 1];
    uint32_t wait_failed;
    uint32_t n_cand;
    uint32_t next_di;   // persistent CTAs: the descriptor taken ahead (its records prefetched to L2)
    unsigned long long base;
    unsigned long long mbar;
};
// (the bitmaps and digit counts are cleared with 16-byte stores)
static_assert(offsetof(GroupSmem<GroupLarge>, u) % 16 == 0 && offsetof(GroupSmem<GroupLarge>, cnt) % 16 == 0 &&
                  offsetof(GroupSmem<GroupSmall>, u) % 16 == 0 && offsetof(GroupSmem<GroupSmall>, cnt) % 16 == 0,
              "grouping shared-memory layout");

__device__ __forceinline__ uint64_t pack_pair(uint64_t a, uint64_t b, int idbits) {
    return a < b ? ((a << idbits) | b) : ((b << idbits) | a);
}

// Groups one bucket. Records of equal hash (record >> idbits) form a run; every pair of
// positions in a run is written as (min id << idbits) | max id.
//   1. a two-bitmap filter over kBitmapBits hash bits keeps only records that can have a
//      partner (every record of a run of >= 2 survives; ~1 in 20 singletons does too); the
//      survivors are collected in any order, one shared atomic per warp;
//   2. the survivors are counting-sorted by kDigitBits further hash bits;
//   3. each survivor checks its digit: it heads a run when no earlier survivor of the digit
//      has its hash, and the run's size is the number with that hash (found once, kept per
//      slot, then written at block-scanned offsets);
//   4. the CTA reserves its output range with one atomic on `cursor` and spreads the pairs
//      over its threads. Entries at or past `cap` are counted but not written, so the caller
//      can grow the buffer to the exact size and run again.
// A bucket with more than kMaxRuns runs is appended to `overflow` (grouped later by sorting).
// With n_desc null, CTA i groups descriptor i (the grid has one CTA per descriptor). Otherwise
// the CTAs are persistent: they take descriptors from a queue (counters[kCntNext]) until the
// device-side count *n_desc (at most overflow_cap) is reached, so the grid needs no host-side
// count (the graph form); each takes its next descriptor one bucket ahead and prefetches that
// bucket's records to L2 while it works on the current one.
constexpr int kCntNext = 7;  // the persistent grouping's queue position

template <class G>
__global__ void __launch_bounds__(G::kThreads, G::kMinCtas) k_bucket_group(const BucketDesc* __restrict__ descs,
                                                                     const uint64_t* __restrict__ buf_a,
                                                                     const uint64_t* __restrict__ buf_b, int idbits,
                                                                     uint64_t* __restrict__ pairs, uint64_t cap,
                                                                     unsigned long long* __restrict__ cursor,
                                                                     unsigned int* __restrict__ errors, int use_tma,
                                                                     BucketDesc* __restrict__ overflow,
                                                                     uint32_t overflow_cap,
                                                                     unsigned int* __restrict__ counters,
                                                                     const unsigned int* __restrict__ n_desc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GroupSmem<G>& S = *reinterpret_cast<GroupSmem<G>*>(smem_raw);
    const uint32_t mbar = smem_u32(&S.mbar);
    if (use_tma && threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const uint32_t count = n_desc ? min(*n_desc, overflow_cap) : gridDim.x;
    uint32_t phase = 0;
    for (uint32_t iter = 0;; iter++, phase ^= 1u) {
    __syncthreads();  // the previous descriptor is done with the shared memory
    if (threadIdx.x == 0)
        S.n_cand = n_desc ? (iter == 0 ? atomicAdd(&counters[kCntNext], 1u) : S.next_di)
                          : (iter == 0 ? blockIdx.x : count);
    __syncthreads();
    const uint32_t di = S.n_cand;
    if (di >= count) return;
    const BucketDesc bd = descs[di];
    const uint32_t n = bd.size;
    const uint64_t* src = (bd.src ? buf_b : buf_a) + bd.start;
    // The bucket goes to shared memory either by one TMA bulk copy (use_tma) or by plain
    // 16-byte loads from all threads. A bulk copy must start on 16 bytes and move a multiple
    // of 16 bytes: both paths copy from the 16-byte boundary at or below the first record (one
    // extra record at most on each side; the record buffers carry 16 bytes of padding).
    const uint32_t lead = (uint32_t)(((uintptr_t)src & 15u) >> 3);
    const uint64_t* src16 = src - lead;
    const uint32_t bytes = ((lead + n) * 8u + 15u) & ~15u;
    if (threadIdx.x == 0) S.wait_failed = 0;
    if (use_tma) {
        if (threadIdx.x == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_u32(&S.rec[0])),
                "l"(src16), "r"(bytes), "r"(mbar)
                : "memory");
        }
    } else {
        const uint4* g = reinterpret_cast<const uint4*>(src16);
        uint4* dd = reinterpret_cast<uint4*>(&S.rec[0]);
        for (uint32_t i = threadIdx.x; i < bytes / 16; i += G::kThreads) dd[i] = __ldg(g + i);
    }
    if (n_desc && threadIdx.x == 0) {
        // persistent CTAs take their next descriptor now and start its records towards L2, so
        // that its copy, one bucket later, does not wait on DRAM
        const uint32_t nd = atomicAdd(&counters[kCntNext], 1u);
        S.next_di = nd;
        if (nd < count) {
            const BucketDesc nbd = descs[nd];
            const uint64_t* nsrc = (nbd.src ? buf_b : buf_a) + nbd.start;
            const uint32_t nlead = (uint32_t)(((uintptr_t)nsrc & 15u) >> 3);
            const uint32_t nbytes = ((nlead + nbd.size) * 8u + 15u) & ~15u;
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(nsrc - nlead), "r"(nbytes) : "memory");
        }
    }
    {
        // both bitmaps and the digit counts cleared with 16-byte stores
        uint4* bm = reinterpret_cast<uint4*>(S.u.bm.seen);
        for (int i = threadIdx.x; i < G::kBitmapWords / 2; i += G::kThreads) bm[i] = make_uint4(0, 0, 0, 0);
        uint4* cn = reinterpret_cast<uint4*>(S.cnt);
        for (int i = threadIdx.x; i < G::kDigits / 4; i += G::kThreads) cn[i] = make_uint4(0, 0, 0, 0);
    }
    if (use_tma && threadIdx.x == 0) {
        // one thread polls the barrier (sleeping between polls); the others wait at __syncthreads
        uint32_t polls = 0;
        while (!mbar_try_wait(mbar, phase)) {
            if (++polls > kWaitLimit) {
                S.wait_failed = 1;
                break;
            }
            __nanosleep(32);
        }
    }
    __syncthreads();
    if (S.wait_failed) {
        // one more bounded wait for the copy to land before the shared memory is released
        if (threadIdx.x == 0) {
            uint32_t polls = 0;
            while (!mbar_try_wait(mbar, phase) && ++polls < kWaitLimit) __nanosleep(64);
            atomicAdd(errors, 1u);
        }
        __syncthreads();
        return;
    }
    const uint64_t* rec = S.rec + lead;
    const uint64_t idmask = (1ull << idbits) - 1ull;

    // 1. bitmap filter; each thread keeps its records' bitmap positions for the second pass
    constexpr int kPerThread = G::kCap / G::kThreads;
    uint32_t pos[kPerThread];
#pragma unroll
    for (int k = 0; k < kPerThread; k++) {
        const uint32_t i = threadIdx.x + (uint32_t)k * G::kThreads;
        pos[k] = 0;
        if (i < n) {
            const uint32_t b = (uint32_t)(rec[i] >> idbits) & (G::kBitmapBits - 1);
            const uint32_t bit = 1u << (b & 31);
            if (atomicOr(&S.u.bm.seen[b >> 5], bit) & bit) atomicOr(&S.u.bm.twice[b >> 5], bit);
            pos[k] = b;
        }
    }
    __syncthreads();
    // candidates in any order: each warp keeps its ballots in registers and counts its hits, the
    // warps' counts are summed in order, then each warp writes its candidates at its offset (no
    // shared counter for all warps to contend on)
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    unsigned masks[kPerThread];
    uint32_t mine = 0;
#pragma unroll
    for (int k = 0; k < kPerThread; k++) {
        const uint32_t i = threadIdx.x + (uint32_t)k * G::kThreads;
        bool hit = false;
        if (i < n) {
            const uint32_t b = pos[k];
            hit = (S.u.bm.twice[b >> 5] >> (b & 31)) & 1u;
        }
        masks[k] = __ballot_sync(0xffffffffu, hit);
        mine += __popc(masks[k]);
    }
    if (lane == 0) S.warp_sums[warp] = mine;
    __syncthreads();
    uint32_t cbase = 0, m = 0;
#pragma unroll
    for (int w = 0; w < G::kThreads / 32; w++) {
        const uint32_t v = S.warp_sums[w];
        cbase += w < (int)warp ? v : 0u;
        m += v;
    }
    const unsigned lt = (1u << lane) - 1u;
    // (each candidate is also counted in its digit of the counting sort below)
#pragma unroll
    for (int k = 0; k < kPerThread; k++) {
        if ((masks[k] >> lane) & 1u) {
            const uint32_t i = threadIdx.x + k * G::kThreads;
            S.cand[cbase + __popc(masks[k] & lt)] = (uint16_t)i;
            atomicAdd(&S.cnt[(uint32_t)(rec[i] >> (idbits + G::kBitmapLog)) & (G::kDigits - 1)], 1u);
        }
        cbase += __popc(masks[k]);
    }
    __syncthreads();  // the bitmaps are dead from here on

    // 2. counting sort of the candidates by kDigitBits hash bits above the bitmap bits (the
    //    digit counts were taken above)
    constexpr int kPer = G::kDigits / G::kThreads;
    {
        const int d0 = threadIdx.x * kPer;
        uint32_t loc[kPer], sum = 0;
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            loc[k] = sum;
            sum += S.cnt[d0 + k];
        }
        uint32_t tot;
        const uint32_t ex = block_scan_ex<uint32_t, G::kThreads>(sum, &tot, S.warp_sums);
#pragma unroll
        for (int k = 0; k < kPer; k++) S.cnt[d0 + k] = ex + loc[k];
    }
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < m; c += G::kThreads) {
        const uint16_t i = S.cand[c];
        const uint32_t p = atomicAdd(&S.cnt[(uint32_t)(rec[i] >> (idbits + G::kBitmapLog)) & (G::kDigits - 1)], 1u);
        S.u.gr.perm[p] = i;
    }
    __syncthreads();
    // now digit dg occupies perm[cnt[dg-1] .. cnt[dg])

    // 3. runs
    auto scan_pos = [&](uint32_t i, uint32_t& size, uint32_t& contiguous) -> bool {
        const uint64_t kv = rec[S.u.gr.perm[i]] >> idbits;
        const uint32_t dg = (uint32_t)(kv >> G::kBitmapLog) & (G::kDigits - 1);
        const uint32_t a = dg == 0 ? 0u : S.cnt[dg - 1], b = S.cnt[dg];
        if (b - a < 2) return false;
        for (uint32_t y = a; y < i; y++)
            if ((rec[S.u.gr.perm[y]] >> idbits) == kv) return false;
        // (four independent loads per step: a long run's head does not wait on one chain)
        uint32_t sz = 1, y = i + 1;
        for (; y + 4 <= b; y += 4) {
            const uint32_t p0 = S.u.gr.perm[y], p1 = S.u.gr.perm[y + 1], p2 = S.u.gr.perm[y + 2],
                           p3 = S.u.gr.perm[y + 3];
            sz += ((rec[p0] >> idbits) == kv) + ((rec[p1] >> idbits) == kv) + ((rec[p2] >> idbits) == kv) +
                  ((rec[p3] >> idbits) == kv);
        }
        for (; y < b; y++) sz += (rec[S.u.gr.perm[y]] >> idbits) == kv;
        size = sz;
        contiguous = (sz == b - a) ? 1u : 0u;
        return sz >= 2;
    };
    // each slot's run word (contiguous << 15 | size for a run head, 0 otherwise) is kept in
    // `cand`, which the counting sort no longer needs, for the second pass
    uint32_t my_runs = 0, my_pairs = 0;
    for (uint32_t i = threadIdx.x; i < m; i += G::kThreads) {
        uint32_t sz, ct;
        uint16_t word = 0;
        if (scan_pos(i, sz, ct)) {
            my_runs++;
            my_pairs += sz * (sz - 1) / 2;
            word = (uint16_t)((ct << 15) | sz);  // size <= G::kCap < 2^15
        }
        S.cand[i] = word;
    }
    // runs (high half) and pairs (low half: a bucket has fewer than 2^32 pairs) in one scan
    unsigned long long tot64;
    const unsigned long long off64 = block_scan_ex<unsigned long long, G::kThreads>(
        ((unsigned long long)my_runs << 32) | my_pairs, &tot64, S.warp_sums64);
    uint32_t run_off = (uint32_t)(off64 >> 32), pair_off = (uint32_t)off64;
    const uint32_t nr = (uint32_t)(tot64 >> 32), total = (uint32_t)tot64;
    if (nr > (uint32_t)kMaxRuns) {  // too many runs to list: the bucket is regrouped by sorting
        if (threadIdx.x == 0) bounded_append(overflow, overflow_cap, counters, kCntFallback, bd);
        continue;
    }
    for (uint32_t i = threadIdx.x; i < m; i += G::kThreads) {  // the same slots as above
        const uint32_t word = S.cand[i];
        if (word) {
            const uint32_t sz = word & 0x7fffu, ct = word >> 15;
            S.u.gr.runs[run_off] = (ct << 31) | (sz << 16) | i;  // head slot < 2^13, size < 2^15
            S.u.gr.poff[run_off] = pair_off;
            run_off++;
            pair_off += sz * (sz - 1) / 2;
        }
    }
    if (threadIdx.x == 0) S.base = atomicAdd(cursor, (unsigned long long)total);
    __syncthreads();
    const uint64_t base = S.base;

    // 4. pair t of the bucket -> run (binary search over the offsets) -> (i, j) inside the run
    for (uint32_t t = threadIdx.x; t < total; t += G::kThreads) {
        uint32_t lo = 0, hi = nr - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (S.u.gr.poff[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const uint32_t run = S.u.gr.runs[lo];
        const uint32_t s = (run >> 16) & 0x7fffu, x = run & 0xffffu;
        const uint32_t l = t - S.u.gr.poff[lo];
        uint32_t i = 0, j = 1;
        if (s > 2) {
            const float b2 = (float)(2 * s - 1);
            int ii = (int)floorf((b2 - sqrtf(b2 * b2 - 8.0f * (float)l)) * 0.5f);
            i = ii < 0 ? 0u : (uint32_t)ii;
            while (i + 1 < s && (uint32_t)tri_row_start(i + 1, s) <= l) i++;
            while (i > 0 && (uint32_t)tri_row_start(i, s) > l) i--;
            j = i + 1 + (l - (uint32_t)tri_row_start(i, s));
        }
        uint32_t pi, pj;
        if (run >> 31) {  // the run fills its digit: members are consecutive slots
            pi = x + i;
            pj = x + j;
        } else {          // members are the slots of the digit with the head's hash
            const uint64_t kv = rec[S.u.gr.perm[x]] >> idbits;
            uint32_t mm = 0, y = x;
            pi = pj = x;
            for (; mm <= j; y++)
                if ((rec[S.u.gr.perm[y]] >> idbits) == kv) {
                    if (mm == i) pi = y;
                    if (mm == j) pj = y;
                    mm++;
                }
        }
        const uint64_t q = base + t;
        if (q < cap)
            pairs[q] = pack_pair(rec[S.u.gr.perm[pi]] & idmask, rec[S.u.gr.perm[pj]] & idmask, idbits);
    }
    }  // descriptors
}

}  // namespace xtn
