// Hash-bucket grouping of deletion variants (the default key-grouping engine).
//
// The sort-based engine orders all V variant records by hash with a multi-pass radix sort
// (about 24 bytes of HBM traffic per record per 8-bit digit). Grouping only needs equal
// hashes to meet, not a global order, so this engine moves each record through HBM once:
//   count    k_bucket_count    per tile of sequences: histogram of the top B1 hash bits
//                              (variants are generated, hashed and counted, not stored)
//   offsets  k_bucket_colscan  per bucket: exclusive prefix over tiles, bucket totals
//   scatter  k_bucket_scatter  the same variants again, each written once as a 64-bit
//                              record (next hash bits | sequence id) into its bucket's range
//   plan     k_bucket_plan     buckets that fit in shared memory go straight to grouping;
//                              larger ones are split by the next hash bits (k_bucket_split)
//   group    k_bucket_group    one CTA per bucket: TMA bulk copy of the bucket into shared
//                              memory, counting sort on 12 hash bits, runs of equal hashes,
//                              every id pair of every run appended to the candidate list
// Buckets that still exceed shared memory after the split (one variant shared by very many
// sequences) are grouped by the sort-based path instead.
#pragma once
#include <cstdint>

#include "xtn_common.cuh"

namespace xtn {

constexpr int kBucketThreads = 1024;   // count/scatter CTAs (one per SM: up to 128 KB of counters)
constexpr int kGroupThreads = 512;
constexpr int kGroupCap = 8192;        // records a grouping CTA holds in shared memory
constexpr int kDigitBits = 12;
constexpr int kDigits = 1 << kDigitBits;
constexpr int kBigGroup = 48;          // runs at least this long are emitted by the whole CTA
constexpr int kMaxBigGroups = 64;
constexpr uint32_t kWaitLimit = 1u << 26;  // bound on mbarrier polls

// Descriptor of one bucket (or sub-bucket) handed to the grouping kernel.
struct BucketDesc {
    uint64_t start;   // first record
    uint32_t size;    // records
    uint32_t src;     // 0: records in buffer A, 1: in buffer B
};

// Split job: bucket `start,size` (buffer A) is divided into 2^bits sub-buckets (buffer B).
struct SplitJob {
    uint64_t start;
    uint32_t size;
    uint32_t bits;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__global__ void __launch_bounds__(kBucketThreads) k_bucket_count(const u128* __restrict__ keys,
                                                                 const uint8_t* __restrict__ klen, int n, int tile, int d,
                                                                 int b1, uint32_t* __restrict__ counts) {
    extern __shared__ uint32_t s_hist[];
    const int nb = 1 << b1;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s_hist[i] = 0;
    __syncthreads();
    const int base = blockIdx.x * tile;
    const int end = min(n, base + tile);
    const int shift = 64 - b1;
    for (int i = base + threadIdx.x; i < end; i += blockDim.x)
        for_each_variant(keys[i], klen[i], d, [&](u128 k) { atomicAdd(&s_hist[key_hash(k) >> shift], 1u); });
    __syncthreads();
    uint32_t* out = counts + (size_t)blockIdx.x * nb;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) out[i] = s_hist[i];
}

// counts/offsets are tile-major [tile][bucket]; offsets become the exclusive prefix over tiles.
__global__ void k_bucket_colscan(const uint32_t* __restrict__ counts, int ntiles, int nb, uint32_t* __restrict__ offsets,
                                 uint32_t* __restrict__ totals) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    uint32_t run = 0;
    for (int t = 0; t < ntiles; t++) {
        uint32_t c = counts[(size_t)t * nb + b];
        offsets[(size_t)t * nb + b] = run;
        run += c;
    }
    totals[b] = run;
}

__global__ void __launch_bounds__(kBucketThreads) k_bucket_scatter(const u128* __restrict__ keys,
                                                                   const uint8_t* __restrict__ klen, int n, int tile, int d,
                                                                   int b1, int idbits, const uint32_t* __restrict__ offsets,
                                                                   const uint64_t* __restrict__ bstart,
                                                                   uint64_t* __restrict__ recs) {
    extern __shared__ uint32_t s_cur[];
    const int nb = 1 << b1;
    const uint32_t* off = offsets + (size_t)blockIdx.x * nb;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s_cur[i] = (uint32_t)bstart[i] + off[i];
    __syncthreads();
    const int base = blockIdx.x * tile;
    const int end = min(n, base + tile);
    const int shift = 64 - b1;
    const uint64_t hi_mask = ~((1ull << idbits) - 1ull);
    for (int i = base + threadIdx.x; i < end; i += blockDim.x) {
        const uint64_t id = (uint64_t)i;
        for_each_variant(keys[i], klen[i], d, [&](u128 k) {
            uint64_t h = key_hash(k);
            uint32_t pos = atomicAdd(&s_cur[h >> shift], 1u);
            recs[pos] = ((h << b1) & hi_mask) | id;
        });
    }
}

// Sorts buckets into "group directly" descriptors and split jobs.
__global__ void k_bucket_plan(const uint64_t* __restrict__ bstart, int nb, uint32_t group_cap,
                              BucketDesc* __restrict__ desc, SplitJob* __restrict__ jobs,
                              unsigned int* __restrict__ counters) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    uint64_t s = bstart[b], e = bstart[b + 1];
    uint32_t size = (uint32_t)(e - s);
    if (size < 2) return;
    if (size <= group_cap) {
        unsigned k = atomicAdd(&counters[0], 1u);
        desc[k] = BucketDesc{s, size, 0};
    } else {
        uint32_t bits = 1;
        while (bits < 10 && ((uint64_t)size >> bits) > (uint64_t)(group_cap / 2)) bits++;
        unsigned k = atomicAdd(&counters[1], 1u);
        jobs[k] = SplitJob{s, size, bits};
        atomicAdd(&counters[2], 1u << bits);
    }
}

// One CTA per split job: histogram of the next `bits` hash bits (the record's top bits),
// prefix, then a scatter into buffer B at the same range. Sub-buckets that fit are listed
// for grouping; larger ones go to the fallback list.
__global__ void __launch_bounds__(1024) k_bucket_split(const SplitJob* __restrict__ jobs, const uint64_t* __restrict__ in,
                                                       uint64_t* __restrict__ out, uint32_t group_cap,
                                                       BucketDesc* __restrict__ desc, BucketDesc* __restrict__ fallback,
                                                       unsigned int* __restrict__ counters) {
    __shared__ uint32_t s_cnt[1024];
    __shared__ uint32_t s_cur[1024];
    const SplitJob job = jobs[blockIdx.x];
    const int nsub = 1 << job.bits;
    const int shift = 64 - (int)job.bits;
    for (int i = threadIdx.x; i < nsub; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();
    const uint64_t* src = in + job.start;
    for (uint32_t i = threadIdx.x; i < job.size; i += blockDim.x) atomicAdd(&s_cnt[src[i] >> shift], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int i = 0; i < nsub; i++) {
            uint32_t c = s_cnt[i];
            s_cur[i] = run;
            if (c >= 2) {
                BucketDesc bd{job.start + run, c, 1};
                if (c <= group_cap) desc[atomicAdd(&counters[0], 1u)] = bd;
                else fallback[atomicAdd(&counters[3], 1u)] = bd;
            }
            run += c;
        }
    }
    __syncthreads();
    uint64_t* dst = out + job.start;
    for (uint32_t i = threadIdx.x; i < job.size; i += blockDim.x) {
        uint64_t r = src[i];
        dst[atomicAdd(&s_cur[r >> shift], 1u)] = r;
    }
}

// Shared-memory layout of k_bucket_group (about 99 KB: two CTAs per SM).
struct GroupSmem {
    uint64_t rec[kGroupCap + 2];  // bucket records (+ alignment slack)
    uint32_t cnt[kDigits];        // counting sort over kDigitBits hash bits
    uint16_t perm[kGroupCap];     // record indexes grouped by digit
    uint32_t big_start[kMaxBigGroups];
    uint32_t big_size[kMaxBigGroups];
    uint64_t big_poff[kMaxBigGroups + 1];
    uint32_t warp_sums32[kGroupThreads / 32 + 1];
    uint64_t warp_sums64[kGroupThreads / 32 + 1];
    unsigned long long base;
    uint32_t n_big;
    uint32_t wait_failed;
    unsigned long long mbar;
};

// Exclusive block scan of one value per thread (kGroupThreads threads).
template <typename T>
__device__ __forceinline__ T group_block_scan(T v, T* total, T* warp_sums) {
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
        T w = lane < kGroupThreads / 32 ? warp_sums[lane] : T(0);
        T winc = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T t = __shfl_up_sync(0xffffffffu, winc, o);
            if (lane >= o) winc += t;
        }
        if (lane < kGroupThreads / 32) warp_sums[lane] = winc - w;
        if (lane == kGroupThreads / 32 - 1) warp_sums[kGroupThreads / 32] = winc;
    }
    __syncthreads();
    T r = inc - v + warp_sums[warp];
    *total = warp_sums[kGroupThreads / 32];
    __syncthreads();
    return r;
}

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

__device__ __forceinline__ uint64_t pack_pair(uint64_t a, uint64_t b, int idbits) {
    return a < b ? ((a << idbits) | b) : ((b << idbits) | a);
}

// Groups one bucket. Records of equal hash (record >> idbits) form a run; every pair of
// positions in a run is written as (min id << idbits) | max id. The CTA reserves its output
// range with one atomic on `cursor`; entries at or past `cap` are counted but not written,
// so the caller can grow the buffer to the exact size and run again.
__global__ void __launch_bounds__(kGroupThreads, 2) k_bucket_group(const BucketDesc* __restrict__ descs,
                                                                     const uint64_t* __restrict__ buf_a,
                                                                     const uint64_t* __restrict__ buf_b, int idbits,
                                                                     uint64_t* __restrict__ pairs, uint64_t cap,
                                                                     unsigned long long* __restrict__ cursor,
                                                                     unsigned int* __restrict__ errors) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GroupSmem& S = *reinterpret_cast<GroupSmem*>(smem_raw);
    const BucketDesc bd = descs[blockIdx.x];
    const uint32_t n = bd.size;
    const uint64_t* src = (bd.src ? buf_b : buf_a) + bd.start;
    // TMA bulk copy of the bucket into shared memory. The source must start on 16 bytes and
    // the size must be a multiple of 16: copy from the 16-byte boundary at or below the first
    // record (one extra record at most on each side; the buffers carry 16 bytes of padding).
    const uint32_t lead = (uint32_t)(((uintptr_t)src & 15u) >> 3);
    const uint64_t* src16 = src - lead;
    const uint32_t bytes = ((lead + n) * 8u + 15u) & ~15u;
    const uint32_t mbar = smem_u32(&S.mbar);
    if (threadIdx.x == 0) {
        S.wait_failed = 0;
        S.n_big = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_u32(&S.rec[0])),
            "l"(src16), "r"(bytes), "r"(mbar)
            : "memory");
    }
    for (int i = threadIdx.x; i < kDigits; i += kGroupThreads) S.cnt[i] = 0;
    __syncthreads();
    {
        uint32_t polls = 0;
        while (!mbar_try_wait(mbar, 0)) {
            if (++polls > kWaitLimit) {
                atomicExch(&S.wait_failed, 1u);
                break;
            }
        }
    }
    __syncthreads();
    if (S.wait_failed) {
        // one more bounded wait for the copy to land before the shared memory is released
        if (threadIdx.x == 0) {
            uint32_t polls = 0;
            while (!mbar_try_wait(mbar, 0) && ++polls < kWaitLimit) {
            }
            atomicAdd(errors, 1u);
        }
        __syncthreads();
        return;
    }
    const uint64_t* rec = S.rec + lead;
    const uint64_t idmask = (1ull << idbits) - 1ull;

    // counting sort by kDigitBits hash bits
    for (uint32_t i = threadIdx.x; i < n; i += kGroupThreads) atomicAdd(&S.cnt[(rec[i] >> idbits) & (kDigits - 1)], 1u);
    __syncthreads();
    constexpr int kPer = kDigits / kGroupThreads;
    const int d0 = threadIdx.x * kPer;
    {
        uint32_t loc[kPer], sum = 0;
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            loc[k] = sum;
            sum += S.cnt[d0 + k];
        }
        uint32_t tot;
        uint32_t ex = group_block_scan<uint32_t>(sum, &tot, S.warp_sums32);
#pragma unroll
        for (int k = 0; k < kPer; k++) S.cnt[d0 + k] = ex + loc[k];
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += kGroupThreads) {
        uint32_t p = atomicAdd(&S.cnt[(rec[i] >> idbits) & (kDigits - 1)], 1u);
        S.perm[p] = (uint16_t)i;
    }
    __syncthreads();
    // now digit dg occupies perm[cnt[dg-1] .. cnt[dg])

    // runs of equal hash inside each of this thread's digits (a digit holds ~2 records)
    uint64_t my_pairs = 0, listed = 0;
    int seen_big = 0;
    for (int k = 0; k < kPer; k++) {
        const int dg = d0 + k;
        const uint32_t a = dg == 0 ? 0u : S.cnt[dg - 1], b = S.cnt[dg];
        if (b - a < 2) continue;
        for (uint32_t x = a + 1; x < b; x++) {
            uint16_t v = S.perm[x];
            uint64_t kv = rec[v] >> idbits;
            uint32_t y = x;
            while (y > a && (rec[S.perm[y - 1]] >> idbits) > kv) {
                S.perm[y] = S.perm[y - 1];
                y--;
            }
            S.perm[y] = v;
        }
        for (uint32_t x = a; x < b;) {
            uint64_t kv = rec[S.perm[x]] >> idbits;
            uint32_t y = x + 1;
            while (y < b && (rec[S.perm[y]] >> idbits) == kv) y++;
            const uint64_t s = y - x;
            if (s >= (uint64_t)kBigGroup && seen_big < 64) {
                uint32_t slot = atomicAdd(&S.n_big, 1u);
                if (slot < (uint32_t)kMaxBigGroups) {
                    S.big_start[slot] = x;
                    S.big_size[slot] = (uint32_t)s;
                    listed |= 1ull << seen_big;
                } else {
                    my_pairs += s * (s - 1) / 2;
                }
                seen_big++;
            } else if (s >= 2) {
                my_pairs += s * (s - 1) / 2;
            }
            x = y;
        }
    }
    __syncthreads();
    const uint32_t n_big = min(S.n_big, (uint32_t)kMaxBigGroups);
    if (threadIdx.x == 0) {
        uint64_t run = 0;
        for (uint32_t g = 0; g < n_big; g++) {
            S.big_poff[g] = run;
            uint64_t s = S.big_size[g];
            run += s * (s - 1) / 2;
        }
        S.big_poff[n_big] = run;
    }
    uint64_t total;
    const uint64_t my_off = group_block_scan<uint64_t>(my_pairs, &total, S.warp_sums64);
    if (threadIdx.x == 0) S.base = atomicAdd(cursor, (unsigned long long)(total + S.big_poff[n_big]));
    __syncthreads();
    const uint64_t base = S.base;

    // runs emitted by their own thread
    uint64_t o = base + my_off;
    seen_big = 0;
    for (int k = 0; k < kPer; k++) {
        const int dg = d0 + k;
        const uint32_t a = dg == 0 ? 0u : S.cnt[dg - 1], b = S.cnt[dg];
        if (b - a < 2) continue;
        for (uint32_t x = a; x < b;) {
            uint64_t kv = rec[S.perm[x]] >> idbits;
            uint32_t y = x + 1;
            while (y < b && (rec[S.perm[y]] >> idbits) == kv) y++;
            const uint32_t s = y - x;
            bool mine = s >= 2;
            if (s >= (uint32_t)kBigGroup && seen_big < 64) {
                if ((listed >> seen_big) & 1ull) mine = false;
                seen_big++;
            }
            if (mine)
                for (uint32_t i = x; i < y; i++) {
                    const uint64_t ai = rec[S.perm[i]] & idmask;
                    for (uint32_t j = i + 1; j < y; j++) {
                        if (o < cap) pairs[o] = pack_pair(ai, rec[S.perm[j]] & idmask, idbits);
                        o++;
                    }
                }
            x = y;
        }
    }
    // listed runs: the whole CTA, pair index t -> (i, j) inside the run
    const uint64_t bo = base + total;
    for (uint32_t g = 0; g < n_big; g++) {
        const uint64_t s = S.big_size[g], x = S.big_start[g];
        const uint64_t np = s * (s - 1) / 2;
        for (uint64_t t = threadIdx.x; t < np; t += kGroupThreads) {
            double b2 = (double)(2 * s - 1);
            int64_t ii = (int64_t)floor((b2 - sqrt(b2 * b2 - 8.0 * (double)t)) * 0.5);
            uint64_t i = ii < 0 ? 0 : (uint64_t)ii;
            while (i + 1 < s && tri_row_start(i + 1, s) <= t) i++;
            while (i > 0 && tri_row_start(i, s) > t) i--;
            const uint64_t j = i + 1 + (t - tri_row_start(i, s));
            const uint64_t q = bo + S.big_poff[g] + t;
            if (q < cap) pairs[q] = pack_pair(rec[S.perm[x + i]] & idmask, rec[S.perm[x + j]] & idmask, idbits);
        }
    }
}

}  // namespace xtn
