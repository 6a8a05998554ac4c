// Device-wide primitives written for this library: exclusive prefix sums and a stable LSD
// radix sort of 64-bit keys. They replace the CUB calls of the reference
// (S/src/cub.cu:80-104,116-124,136-173) on this path.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

namespace xtn {

// ------------------------------------------------------------------ launch accounting
// Every kernel launch of the library goes through XTN_LAUNCH, which counts it and, when
// profiling is on, brackets it with a pair of CUDA events on the launching stream so the
// caller can read per-kernel device time after the run.
struct KernelProfiler {
    bool on = false;
    std::string only;  // when set, only launches of this kernel name are bracketed
    bool skipping = false;
    int64_t launches = 0;
    struct Rec {
        const char* name;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    size_t used = 0;
    cudaStream_t stream = nullptr;
    void reset(cudaStream_t s) {
        stream = s;
        used = 0;
        launches = 0;
    }
    void begin(const char* name) {
        launches++;
        skipping = !on || (!only.empty() && only != name);
        if (skipping) return;
        if (used == recs.size()) {
            Rec r{name, nullptr, nullptr};
            cudaEventCreate(&r.a);
            cudaEventCreate(&r.b);
            recs.push_back(r);
        }
        recs[used].name = name;
        cudaEventRecord(recs[used].a, stream);
    }
    void end() {
        if (skipping) return;
        cudaEventRecord(recs[used].b, stream);
        used++;
    }
    ~KernelProfiler() {
        for (auto& r : recs) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
    }
};

inline KernelProfiler*& current_profiler() {
    static thread_local KernelProfiler* p = nullptr;
    return p;
}

#define XTN_LAUNCH(name, ...)                                  \
    do {                                                       \
        ::xtn::KernelProfiler* pr_ = ::xtn::current_profiler(); \
        if (pr_) pr_->begin(name);                             \
        __VA_ARGS__;                                           \
        if (pr_) pr_->end();                                   \
    } while (0)

constexpr int kScanBlock = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Relaxed loads and stores of status words that other CTAs poll (gpu scope, no L1 caching).
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Exclusive scan of one value per thread across the block; returns the block total in *total.
template <typename T, int BLOCK>
__device__ __forceinline__ T block_exclusive_scan(T v, T* total) {
    __shared__ T warp_sums[BLOCK / 32 + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = warp_inclusive_scan(v);
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < BLOCK / 32 ? warp_sums[lane] : T(0);
        T winc = warp_inclusive_scan(w);
        if (lane < BLOCK / 32) warp_sums[lane] = winc - w;
        if (lane == BLOCK / 32 - 1) warp_sums[BLOCK / 32] = winc;
    }
    __syncthreads();
    T r = inc - v + warp_sums[warp];
    *total = warp_sums[BLOCK / 32];
    __syncthreads();
    return r;
}

template <typename In, typename Out>
__global__ void __launch_bounds__(kScanBlock) k_scan_reduce(const In* __restrict__ in, Out* __restrict__ sums, int64_t n) {
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    Out s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + (int64_t)k * kScanBlock + threadIdx.x;
        if (i < n) s += (Out)in[i];
    }
    __shared__ Out red[kScanBlock / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        Out t = threadIdx.x < kScanBlock / 32 ? red[threadIdx.x] : Out(0);
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) sums[blockIdx.x] = t;
    }
}

// out[i] = offset[tile] + sum(in[0..i) within the tile); out[n] = grand total when the
// caller passes n_out = n + 1 (the last tile writes it).
template <typename In, typename Out>
__global__ void __launch_bounds__(kScanBlock) k_scan_tiles(const In* __restrict__ in, Out* __restrict__ out,
                                                           const Out* __restrict__ tile_offsets, int64_t n, bool write_total) {
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    Out v[kScanItems];
    Out s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + k;
        v[k] = i < n ? (Out)in[i] : Out(0);
        s += v[k];
    }
    Out total;
    Out ex = block_exclusive_scan<Out, kScanBlock>(s, &total);
    Out off = tile_offsets ? tile_offsets[blockIdx.x] : Out(0);
    Out run = off + ex;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
    if (write_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = off + total;
}

// Scratch requirement (in Out elements) for scan_exclusive over n items.
inline int64_t scan_scratch_elems(int64_t n) {
    int64_t total = 0;
    while (n > kScanTile) {
        int64_t t = (n + kScanTile - 1) / kScanTile;
        total += 2 * t + 1;
        n = t;
    }
    return total + 1;
}

// Exclusive scan of n items into out[0..n), with out[n] = total. `scratch` holds
// scan_scratch_elems(n) Out elements. Asynchronous on `stream`.
template <typename In, typename Out>
void scan_exclusive(const In* in, Out* out, int64_t n, Out* scratch, cudaStream_t stream) {
    if (n <= 0) {
        cudaMemsetAsync(out, 0, sizeof(Out), stream);
        return;
    }
    int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        XTN_LAUNCH("scan_tiles", (k_scan_tiles<In, Out><<<1, kScanBlock, 0, stream>>>(in, out, nullptr, n, true)));
        return;
    }
    Out* sums = scratch;
    Out* offs = scratch + tiles;
    XTN_LAUNCH("scan_reduce", (k_scan_reduce<In, Out><<<(unsigned)tiles, kScanBlock, 0, stream>>>(in, sums, n)));
    scan_exclusive<Out, Out>(sums, offs, tiles, scratch + 2 * tiles + 1, stream);
    XTN_LAUNCH("scan_tiles", (k_scan_tiles<In, Out><<<(unsigned)tiles, kScanBlock, 0, stream>>>(in, out, offs, n, true)));
}

// Single-pass exclusive scan (decoupled look-back, as in Merrill & Garland, "Single-pass
// parallel prefix scan with decoupled look-back", 2016): a CTA takes the next tile in start order
// (an atomic ticket), publishes its tile total in a status word, and warp 0 sums the totals of
// earlier tiles 32 at a time, back to the nearest inclusive prefix, before publishing its own.
// A tile waits only for tiles taken earlier by running CTAs, which publish before they look
// back, so the waits end; each is still bounded (poll_limit rounds, kScanPollLimit by default),
// after which *err is incremented and the tile continues with the sum it has (the host reports
// the error and discards the result). One launch instead of scan_exclusive's three or more;
// `status` holds scan_1p_words(n) words that the call clears first. Status word: bits 62-63
// flag (1: tile total, 2: inclusive prefix), bits 0-61 the value. withhold_tile0 != 0 makes tile
// 0 skip publishing its prefix: a status word that nothing sets, so that a test can make the
// later tiles' bounded waits run out and check that the error reaches the caller.
constexpr unsigned long long kScanFlagTotal = 1ull << 62;
constexpr unsigned long long kScanFlagPrefix = 2ull << 62;
constexpr unsigned long long kScanValueMask = (1ull << 62) - 1ull;
constexpr uint32_t kScanPollLimit = 1u << 22;

inline int64_t scan_1p_words(int64_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

// n_dev (graph form, may be null): n is a capacity and the item count is read on the device;
// tiles past it leave at once (no later tile is real) and the last real tile writes out[n].
template <typename In, typename Out>
__global__ void __launch_bounds__(kScanBlock) k_scan_1p(const In* __restrict__ in, Out* __restrict__ out, int64_t n,
                                                        unsigned long long* __restrict__ status,
                                                        unsigned int* __restrict__ err, uint32_t poll_limit,
                                                        int withhold_tile0, const unsigned long long* __restrict__ n_dev) {
    __shared__ uint32_t s_tile;
    __shared__ Out s_excl;
    unsigned int* ticket = reinterpret_cast<unsigned int*>(status);  // word 0; tiles from word 1
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    uint32_t last_tile = gridDim.x - 1;
    if (n_dev) {
        n = (int64_t)min((unsigned long long)n, *n_dev);
        last_tile = n > 0 ? (uint32_t)((n - 1) / kScanTile) : 0u;
        if (tile > last_tile) return;
    }
    const int64_t base = (int64_t)tile * kScanTile + (int64_t)threadIdx.x * kScanItems;
    Out v[kScanItems];
    Out sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        const int64_t i = base + k;
        v[k] = i < n ? (Out)in[i] : Out(0);
        sum += v[k];
    }
    Out total;
    const Out ex = block_exclusive_scan<Out, kScanBlock>(sum, &total);
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        unsigned long long* words = status + 1;
        Out excl = 0;
        if (tile == 0) {
            if (lane == 0 && !withhold_tile0) st_relaxed_u64(words, kScanFlagPrefix | (unsigned long long)total);
        } else {
            if (lane == 0) st_relaxed_u64(words + tile, kScanFlagTotal | (unsigned long long)total);
            uint32_t polls = 0;
            for (int64_t j = (int64_t)tile - 1; j >= 0; j -= 32) {
                const int64_t t = j - lane;  // lane 0 reads the nearest tile
                unsigned long long w = t >= 0 ? ld_relaxed_u64(words + t) : kScanFlagPrefix;
                while (__any_sync(0xffffffffu, (w >> 62) == 0ull) && ++polls <= poll_limit) {
                    if (polls > 64) __nanosleep(64);
                    if ((w >> 62) == 0ull) w = ld_relaxed_u64(words + t);
                }
                if (polls > poll_limit) {
                    if (lane == 0) atomicAdd(err, 1u);
                    break;
                }
                const unsigned pm = __ballot_sync(0xffffffffu, (w >> 62) == 2ull);
                const int stop = pm ? __ffs(pm) - 1 : 31;  // nearest inclusive prefix
                Out part = lane <= stop ? (Out)(w & kScanValueMask) : Out(0);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
                excl += __shfl_sync(0xffffffffu, part, 0);
                if (pm) break;
            }
            if (lane == 0) st_relaxed_u64(words + tile, kScanFlagPrefix | (unsigned long long)(excl + total));
        }
        if (lane == 0) s_excl = excl;
    }
    __syncthreads();
    Out run = s_excl + ex;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        const int64_t i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
    if (tile == last_tile && threadIdx.x == 0) out[n] = s_excl + total;
}

// Exclusive scan of n items into out[0..n), with out[n] = total, in one launch (plus the clear
// of `status`). Asynchronous on `stream`.
template <typename In, typename Out>
void scan_exclusive_1p(const In* in, Out* out, int64_t n, unsigned long long* status, unsigned int* err,
                       cudaStream_t stream, uint32_t poll_limit = kScanPollLimit, int withhold_tile0 = 0,
                       const unsigned long long* n_dev = nullptr) {
    if (n_dev) {  // graph form: always the look-back kernel, sized for n items at most
        const int64_t tiles = std::max<int64_t>(1, (n + kScanTile - 1) / kScanTile);
        cudaMemsetAsync(status, 0, sizeof(unsigned long long) * (tiles + 1), stream);
        XTN_LAUNCH("scan_1p", (k_scan_1p<In, Out><<<(unsigned)tiles, kScanBlock, 0, stream>>>(
                                  in, out, std::max<int64_t>(n, 1), status, err, poll_limit, 0, n_dev)));
        return;
    }
    if (n <= 0) {
        cudaMemsetAsync(out, 0, sizeof(Out), stream);
        return;
    }
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        XTN_LAUNCH("scan_tiles", (k_scan_tiles<In, Out><<<1, kScanBlock, 0, stream>>>(in, out, nullptr, n, true)));
        return;
    }
    cudaMemsetAsync(status, 0, sizeof(unsigned long long) * scan_1p_words(n), stream);
    XTN_LAUNCH("scan_1p", (k_scan_1p<In, Out><<<(unsigned)tiles, kScanBlock, 0, stream>>>(in, out, n, status, err,
                                                                                          poll_limit, withhold_tile0,
                                                                                          nullptr)));
}

// ------------------------------------------------------------------ LSD radix sort (u64 keys)
// One pass = upsweep (per-tile digit counts) + exclusive scan over the digit-major count
// matrix + downsweep (stable rank inside the tile with warp match, reorder in shared
// memory, coalesced write of each digit run). Keys carry their payload in the low bits.
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;

__global__ void __launch_bounds__(kSortThreads) k_radix_upsweep(const uint64_t* __restrict__ keys, int64_t n, int shift,
                                                                uint32_t* __restrict__ counts, int64_t ntiles) {
    __shared__ uint32_t hist[kRadix];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int k = 0; k < kSortItems; k++) {
        int64_t i = base + (int64_t)k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&hist[(keys[i] >> shift) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    counts[(int64_t)threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

__global__ void __launch_bounds__(kSortThreads) k_radix_downsweep(const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                                                                  int64_t n, int shift, const uint32_t* __restrict__ offsets,
                                                                  int64_t ntiles) {
    __shared__ uint64_t s_keys[kSortTile];
    __shared__ uint32_t s_cnt[kSortWarps][kRadix + 1];
    __shared__ uint32_t s_start[kRadix];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * (kRadix + 1); i += kSortThreads) (&s_cnt[0][0])[i] = 0;
    __syncthreads();

    const int64_t tile_base = (int64_t)blockIdx.x * kSortTile;
    const int64_t valid64 = n - tile_base;
    const int valid = valid64 > kSortTile ? kSortTile : (int)valid64;
    const unsigned lt = (1u << lane) - 1u;
    uint64_t key[kSortItems];
    uint32_t rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
        int pos = warp * (32 * kSortItems) + k * 32 + lane;  // warp-contiguous tile order
        bool ok = pos < valid;
        uint64_t kv = ok ? in[tile_base + pos] : 0ull;
        unsigned dg = ok ? (unsigned)((kv >> shift) & (kRadix - 1)) : (unsigned)kRadix;
        unsigned peers = __match_any_sync(0xffffffffu, dg);
        int leader = __ffs(peers) - 1;
        uint32_t before = 0;
        if (lane == leader) {
            before = s_cnt[warp][dg];
            s_cnt[warp][dg] = before + __popc(peers);
        }
        before = __shfl_sync(0xffffffffu, before, leader);
        key[k] = kv;
        rank[k] = before + __popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix over warps; then exclusive scan over digits
    uint32_t tot = 0;
    {
        const int d = threadIdx.x;  // kSortThreads == kRadix
#pragma unroll
        for (int w = 0; w < kSortWarps; w++) {
            uint32_t c = s_cnt[w][d];
            s_cnt[w][d] = tot;
            tot += c;
        }
    }
    uint32_t all;
    uint32_t start = block_exclusive_scan<uint32_t, kSortThreads>(tot, &all);
    s_start[threadIdx.x] = start;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; k++) {
        int pos = warp * (32 * kSortItems) + k * 32 + lane;
        if (pos < valid) {
            unsigned dg = (unsigned)((key[k] >> shift) & (kRadix - 1));
            s_keys[s_start[dg] + s_cnt[warp][dg] + rank[k]] = key[k];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < valid; i += kSortThreads) {
        uint64_t kv = s_keys[i];
        unsigned dg = (unsigned)((kv >> shift) & (kRadix - 1));
        out[(int64_t)offsets[(int64_t)dg * ntiles + blockIdx.x] + (i - s_start[dg])] = kv;
    }
}

inline int64_t radix_tiles(int64_t n) { return (n + kSortTile - 1) / kSortTile; }

// Scratch (u32 elements) for radix_sort_u64 over n keys.
inline int64_t radix_scratch_elems(int64_t n) {
    int64_t m = radix_tiles(n) * kRadix;
    return 2 * (m + 1) + scan_scratch_elems(m + 1);
}

// Sorts keys[0..n) by bits [lo_bit, hi_bit), stable. Ping-pongs between `keys` and `alt`;
// returns the buffer that holds the result.
inline uint64_t* radix_sort_u64(uint64_t* keys, uint64_t* alt, int64_t n, int lo_bit, int hi_bit, uint32_t* scratch,
                                cudaStream_t stream, const char* up_name = "radix_upsweep",
                                const char* down_name = "radix_downsweep") {
    if (n <= 1 || hi_bit <= lo_bit) return keys;
    const int64_t ntiles = radix_tiles(n);
    const int64_t m = ntiles * kRadix;
    uint32_t* counts = scratch;
    uint32_t* offsets = scratch + (m + 1);
    uint32_t* sscratch = scratch + 2 * (m + 1);
    uint64_t* src = keys;
    uint64_t* dst = alt;
    for (int shift = lo_bit; shift < hi_bit; shift += kRadixBits) {
        XTN_LAUNCH(up_name, k_radix_upsweep<<<(unsigned)ntiles, kSortThreads, 0, stream>>>(src, n, shift, counts, ntiles));
        scan_exclusive<uint32_t, uint32_t>(counts, offsets, m, sscratch, stream);
        XTN_LAUNCH(down_name, k_radix_downsweep<<<(unsigned)ntiles, kSortThreads, 0, stream>>>(src, dst, n, shift, offsets, ntiles));
        uint64_t* t = src;
        src = dst;
        dst = t;
    }
    return src;
}

// ------------------------------------------------------------------ single-sweep LSD radix sort
// The passes of radix_sort_u64 with each pass's count kernel and count-matrix scan replaced by
// a chained scan (Adinets & Merrill, "Onesweep: a faster least significant digit radix sort
// for GPUs", 2022):
//   1. k_onesweep_hist reads the keys once and counts every pass's digit at the same time; the
//      last CTA to finish turns the counts into each pass's digit starts;
//   2. per pass, k_onesweep_pass: a CTA takes the next tile in start order (an atomic ticket),
//      ranks the tile's keys by digit, publishes its per-digit counts in a status word per
//      (tile, digit), sums the counts of all earlier tiles by looking back through their
//      status words (decoupled look-back) and writes each digit run at its global position.
// A tile only waits for tiles whose tickets were taken earlier, by CTAs already running, and
// those publish their counts before they look back themselves, so every wait ends; each is
// still bounded (kOsPollLimit polls), after which the CTA counts an error in *err and goes on
// with the sum it has (the host reports the error and discards the result).
// Status word: bits 62-63 flag (1: this tile's count, 2: the count of tiles 0..this one),
// bits 32-61 epoch (a per-pass tag: words of earlier passes read as unset, so the array is
// never cleared between passes), bits 0-31 the count.
constexpr int kOsMaxPasses = 8;
// A pass's tile: 16 keys per thread (4096 per CTA, three CTAs per SM); 8 keys per thread and
// five CTAs per SM took 0.076 ms per pass for the 10M search's 5.2M distinct pairs.
constexpr int kOsItems = 16;
constexpr int kOsTile = kSortThreads * kOsItems;
inline int64_t os_tiles(int64_t n) { return (n + kOsTile - 1) / kOsTile; }
constexpr uint32_t kOsPollLimit = 1u << 22;
constexpr uint32_t kOsMaxEpoch = (1u << 30) - 1u;
constexpr unsigned long long kOsFlagCount = 1ull << 62;
constexpr unsigned long long kOsFlagPrefix = 2ull << 62;

// Scratch of one sort (u32 words): digit starts [passes][256], then the counts [passes][256],
// a ticket per pass and the finished-CTA counter, which are cleared before every sort.
constexpr int kOsStartWords = kOsMaxPasses * kRadix;
constexpr int kOsClearWords = kOsMaxPasses * kRadix + kOsMaxPasses + 1;
constexpr int kOsScratchWords = kOsStartWords + kOsClearWords;

__global__ void __launch_bounds__(kSortThreads) k_onesweep_hist(const uint64_t* __restrict__ keys, int64_t n, int lo_bit,
                                                                int passes, uint32_t* __restrict__ dstart,
                                                                uint32_t* __restrict__ counts,
                                                                unsigned int* __restrict__ done,
                                                                const unsigned long long* __restrict__ n_dev) {
    __shared__ uint32_t h[kOsMaxPasses][kRadix];
    __shared__ int last;
    if (n_dev) n = (int64_t)min((unsigned long long)n, *n_dev);  // graph form: count on the device
#pragma unroll
    for (int p = 0; p < kOsMaxPasses; p++) h[p][threadIdx.x] = 0;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * kSortThreads;
    for (int64_t i = (int64_t)blockIdx.x * kSortThreads + threadIdx.x; i < n; i += stride) {
        const uint64_t k = keys[i] >> lo_bit;
        for (int p = 0; p < passes; p++) atomicAdd(&h[p][(k >> (kRadixBits * p)) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    for (int p = 0; p < passes; p++) {
        const uint32_t v = h[p][threadIdx.x];
        if (v) atomicAdd(&counts[p * kRadix + threadIdx.x], v);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int p = 0; p < passes; p++) {
        uint32_t tot;
        const uint32_t v = __ldcg(&counts[p * kRadix + threadIdx.x]);
        dstart[p * kRadix + threadIdx.x] = block_exclusive_scan<uint32_t, kSortThreads>(v, &tot);
    }
}

__global__ void __launch_bounds__(kSortThreads, 3) k_onesweep_pass(const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                                                                int64_t n, int shift, const uint32_t* __restrict__ dstart,
                                                                unsigned long long* __restrict__ status, uint32_t epoch,
                                                                unsigned int* __restrict__ ticket,
                                                                unsigned int* __restrict__ err,
                                                                const unsigned long long* __restrict__ n_dev) {
    __shared__ uint64_t s_keys[kOsTile];
    __shared__ uint32_t s_cnt[kSortWarps][kRadix + 1];
    __shared__ uint32_t s_start[kRadix];
    __shared__ uint32_t s_base[kRadix];
    __shared__ uint32_t s_tile;
    __shared__ int s_failed;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        s_tile = atomicAdd(ticket, 1u);
        s_failed = 0;
    }
    for (int i = threadIdx.x; i < kSortWarps * (kRadix + 1); i += kSortThreads) (&s_cnt[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const int64_t tile_base = (int64_t)tile * kOsTile;
    // graph form: the grid covers n keys at most and the count is read on the device; tiles past
    // it leave before publishing (no later tile is real, so none waits for them)
    if (n_dev) {
        n = (int64_t)min((unsigned long long)n, *n_dev);
        if (tile_base >= n) return;
    }
    const int64_t valid64 = n - tile_base;
    const int valid = valid64 > kOsTile ? kOsTile : (int)valid64;
    const unsigned lt = (1u << lane) - 1u;
    uint64_t key[kOsItems];
    uint32_t rank[kOsItems];
#pragma unroll
    for (int k = 0; k < kOsItems; k++) {
        const int pos = warp * (32 * kOsItems) + k * 32 + lane;  // warp-contiguous tile order
        const bool ok = pos < valid;
        const uint64_t kv = ok ? in[tile_base + pos] : 0ull;
        const unsigned dg = ok ? (unsigned)((kv >> shift) & (kRadix - 1)) : (unsigned)kRadix;
        const unsigned peers = __match_any_sync(0xffffffffu, dg);
        const int leader = __ffs(peers) - 1;
        uint32_t before = 0;
        if (lane == leader) {
            before = s_cnt[warp][dg];
            s_cnt[warp][dg] = before + __popc(peers);
        }
        before = __shfl_sync(0xffffffffu, before, leader);
        key[k] = kv;
        rank[k] = before + __popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();
    const int d = threadIdx.x;  // kSortThreads == kRadix: one digit per thread
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
        const uint32_t c = s_cnt[w][d];
        s_cnt[w][d] = tot;
        tot += c;
    }
    // publish this tile's counts, then look back one predecessor at a time until an inclusive
    // count is met (tile 0 always publishes one), then publish this tile's inclusive count
    unsigned long long* mine = status + (size_t)tile * kRadix + d;
    const unsigned long long tag = (unsigned long long)epoch << 32;
    uint32_t excl = 0;
    if (tile == 0) {
        st_relaxed_u64(mine, kOsFlagPrefix | tag | tot);
    } else {
        st_relaxed_u64(mine, kOsFlagCount | tag | tot);
        const unsigned long long* q = mine - kRadix;
        uint32_t polls = 0;
        for (int64_t j = (int64_t)tile - 1;;) {
            const unsigned long long w = ld_relaxed_u64(q);
            if ((w >> 62) == 0ull || (uint32_t)((w >> 32) & kOsMaxEpoch) != epoch) {
                if (++polls > kOsPollLimit) {
                    atomicAdd(err, 1u);
                    s_failed = 1;
                    break;
                }
                if (polls > 64) __nanosleep(64);
                continue;
            }
            excl += (uint32_t)w;
            if ((w >> 62) == 2ull) break;
            if (--j < 0) {  // past tile 0 without an inclusive count: cannot happen, but never loops
                atomicAdd(err, 1u);
                s_failed = 1;
                break;
            }
            q -= kRadix;
        }
        st_relaxed_u64(mine, kOsFlagPrefix | tag | (excl + tot));
    }
    uint32_t all;
    const uint32_t start = block_exclusive_scan<uint32_t, kSortThreads>(tot, &all);
    s_start[d] = start;
    s_base[d] = dstart[d] + excl - start;  // global index of local slot i of digit d: s_base[d] + i
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kOsItems; k++) {
        const int pos = warp * (32 * kOsItems) + k * 32 + lane;
        if (pos < valid) {
            const unsigned dg = (unsigned)((key[k] >> shift) & (kRadix - 1));
            s_keys[s_start[dg] + s_cnt[warp][dg] + rank[k]] = key[k];
        }
    }
    __syncthreads();
    if (s_failed) return;  // this tile's positions are unknown: nothing is written
    for (int i = threadIdx.x; i < valid; i += kSortThreads) {
        const uint64_t kv = s_keys[i];
        const unsigned dg = (unsigned)((kv >> shift) & (kRadix - 1));
        const uint32_t at = s_base[dg] + (uint32_t)i;
        if (at < (uint64_t)n) out[at] = kv;
    }
}

// Status words a single-sweep sort of n keys uses.
inline int64_t onesweep_status_words(int64_t n) { return os_tiles(n) * kRadix; }

// Same contract as radix_sort_u64, for n < 2^32 and at most kOsMaxPasses passes. `scratch`
// holds kOsScratchWords u32; `status` onesweep_status_words(n) words, all of whose epochs are
// below *epoch + 1 (zero-filled at allocation); *epoch advances by one per pass, and when it
// would pass kOsMaxEpoch the whole status array (status_cap words) is cleared and it restarts.
// *err counts look-back waits that gave up.
// n_dev (graph form, may be null): n is a capacity, the key count is read on the device, and
// the status words are cleared by the call (a replayed graph repeats its epochs).
inline uint64_t* onesweep_sort_u64(uint64_t* keys, uint64_t* alt, int64_t n, int lo_bit, int hi_bit, uint32_t* scratch,
                                   unsigned long long* status, int64_t status_cap, uint32_t* epoch, unsigned int* err,
                                   int sms, cudaStream_t stream, const char* hist_name, const char* pass_name,
                                   const unsigned long long* n_dev = nullptr) {
    if ((!n_dev && n <= 1) || hi_bit <= lo_bit) return keys;
    const int passes = (hi_bit - lo_bit + kRadixBits - 1) / kRadixBits;
    const int64_t ntiles = os_tiles(n);
    uint32_t* dstart = scratch;
    uint32_t* counts = scratch + kOsStartWords;
    unsigned int* tickets = counts + kOsMaxPasses * kRadix;
    unsigned int* done = tickets + kOsMaxPasses;
    cudaMemsetAsync(counts, 0, sizeof(uint32_t) * kOsClearWords, stream);
    if (n_dev) {
        cudaMemsetAsync(status, 0, sizeof(unsigned long long) * std::min<int64_t>(status_cap, ntiles * kRadix), stream);
        *epoch = 0;
    } else if (*epoch + (uint32_t)passes > kOsMaxEpoch) {
        cudaMemsetAsync(status, 0, sizeof(unsigned long long) * status_cap, stream);
        *epoch = 0;
    }
    const int64_t hist_blocks = std::max<int64_t>(1, std::min<int64_t>((n + kSortTile - 1) / kSortTile, (int64_t)sms * 8));
    XTN_LAUNCH(hist_name, k_onesweep_hist<<<(unsigned)hist_blocks, kSortThreads, 0, stream>>>(keys, n, lo_bit, passes, dstart,
                                                                                           counts, done, n_dev));
    uint64_t* src = keys;
    uint64_t* dst = alt;
    for (int p = 0; p < passes; p++) {
        *epoch += 1;
        XTN_LAUNCH(pass_name, k_onesweep_pass<<<(unsigned)std::max<int64_t>(1, ntiles), kSortThreads, 0, stream>>>(
                                  src, dst, n, lo_bit + kRadixBits * p, dstart + p * kRadix, status, *epoch,
                                  tickets + p, err, n_dev));
        uint64_t* t = src;
        src = dst;
        dst = t;
    }
    return src;
}

}  // namespace xtn
