// B200 (sm_100a) symmetric-deletion neighbour search: kernels, host orchestration and the
// C ABI declared in include/xtn_b200.h.
//
// Pipeline for nearest-neighbour mode (reference stages in S/src/xtn.cu:311-473):
//   check    k_check_lengths every sequence 1..500 residues (device-resident inputs)
//   pack     k_pack          first 18 residues -> 128-bit key, run masks, variant count and
//                            the 19-word key table of the polynomial variant hash
//   scan                     variant offsets
//   group    bucket engine   (xtn_bucket.cuh) first-level buckets, split, grouping in shared
//                            memory: every id pair of every run of equal variant hashes,
//                            packed (min << b) | max; or the sort engine (engine = 1): k_gen,
//                            radix_sort_u64, k_find_groups, k_emit
//   dedup    k_pair_dedup    hash set of candidate pairs in HBM; the distinct ones listed
//   sort     onesweep_sort_u64 / radix_sort_u64  distinct pairs in (x, y) order
//   verify   k_verify_t      x != y, Levenshtein (Myers) / Hamming on the full strings, keep
//                            dist <= d (S/src/kernel.cu:359-392)
//   compact  k_compact       sorted (x, y, dist) output
// Everything stays in device memory; the plain form reads a few scalars back to size buffers,
// the graph form none. Larger inputs run in rounds over ranges of first-level buckets.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/xtn_b200.h"
#include "xtn_common.cuh"
#include "xtn_prims.cuh"
#include "xtn_bucket.cuh"

namespace xtn {

// ------------------------------------------------------------------ errors
static thread_local std::string t_err;
static void set_err(const std::string& s) { t_err = s; }

#define XTN_CK(call)                                                                              \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            set_err(std::string(#call) + " failed: " + cudaGetErrorString(e_));                 \
            return e_ == cudaErrorMemoryAllocation ? XTN_ERR_NOMEM : XTN_ERR_CUDA;                \
        }                                                                                         \
    } while (0)

#define XTN_TRY(expr)             \
    do {                          \
        int r_ = (expr);          \
        if (r_ != XTN_SUCCESS) return r_; \
    } while (0)

// ------------------------------------------------------------------ kernels
constexpr int kThreads = 256;

// Packs each sequence's key; with tab != nullptr also writes its key_table (kTabLen words).
// Each warp builds its 32 tables in shared memory (rows of an odd number of words, so the
// lanes' 8-byte stores fall in distinct banks) and stores them with consecutive lanes on
// consecutive words.
constexpr int kPackThreads = 128;
constexpr int kPackRow = kTabLen | 1;

__global__ void __launch_bounds__(kPackThreads) k_pack(const uint8_t* __restrict__ chars, const uint32_t* __restrict__ offs,
                                                       const int32_t* __restrict__ rows, int n, int d,
                                                       u128* __restrict__ keys, uint8_t* __restrict__ klen,
                                                       uint32_t* __restrict__ vcnt, uint64_t* __restrict__ runinfo,
                                                       uint64_t* __restrict__ tab) {
    __shared__ uint64_t s_tab[kPackThreads / 32][32 * kPackRow];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool live = i < n;
    u128 v = 0;
    if (live) {
        int r = rows ? rows[i] : i;
        uint32_t s = offs[r];
        // lengths are validated by k_check_lengths before the host uses anything computed
        // here; the clamp keeps an invalid one from steering the loop below
        const uint32_t L = offs[r + 1] - s;
        int Lk = L < (uint32_t)kKeyLen ? (int)L : kKeyLen;
        // the key's two 64-bit words (key_words), built with 64-bit shifts
        uint64_t wa = 0, wb = 0;
        for (int j = 0; j < Lk; j++) {
            const uint64_t code = (uint64_t)code_of(chars[s + j]);
            if (j < 12) wa |= code << (55 - 5 * j);
            else wb |= code << (25 - 5 * (j - 12));
        }
        v = ((u128)wa << 68) | ((u128)wb << 38);
        keys[i] = v;
        klen[i] = (uint8_t)Lk;
        vcnt[i] = (uint32_t)variant_count(v, Lk, d);
        runinfo[i] = key_run_info(v, Lk);
    }
    if (!tab) return;
    uint64_t* row = s_tab[w] + lane * kPackRow;
    if (live) key_table(v, [&](int slot, uint64_t x) { row[slot] = x; });
    __syncwarp();
    const int i0 = i - lane;
    const int cnt = min(32, n - i0);
    if (cnt <= 0) return;
    uint64_t* dst = tab + (size_t)i0 * kTabLen;
    for (int k = lane; k < cnt * kTabLen; k += 32) dst[k] = s_tab[w][(k / kTabLen) * kPackRow + k % kTabLen];
}

// Device-side check of caller-provided offsets (the device-resident entry points never see
// them on the host): every sequence must have 1..kMaxInputLength residues, as check_offsets
// requires on the host path. *first_bad (preset to 0xffffffff) receives the smallest bad
// index. Kernels that index by length (the verification's DP column, in particular) run only
// after the host has read this word.
__global__ void k_check_lengths(const uint32_t* __restrict__ offs, const int32_t* __restrict__ rows, int n,
                                unsigned int* __restrict__ first_bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = rows ? rows[i] : i;
    const uint32_t a = offs[r], b = offs[r + 1];
    if (b <= a || b - a > (uint32_t)kMaxInputLength) atomicMin(first_bad, (unsigned int)i);
}

// One thread per sequence writes its variant records at voff[i]; d <= 2 hashes come from
// the key tables when given.
__global__ void k_gen(const u128* __restrict__ keys, const uint8_t* __restrict__ klen,
                      const uint64_t* __restrict__ runinfo, const uint64_t* __restrict__ tab,
                      const uint64_t* __restrict__ voff, int n, int d, int idbits, uint64_t* __restrict__ recs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t hi_mask = ~((1ull << idbits) - 1ull);
    uint64_t o = voff[i];
    const uint64_t id = (uint64_t)i;
    if (tab && d <= 2)
        for_each_hash(tab + (size_t)i * kTabLen, klen[i], runinfo[i], d,
                      [&](uint64_t h) { recs[o++] = (h & hi_mask) | id; });
    else
        for_each_variant(keys[i], klen[i], d, [&](u128 k) { recs[o++] = (key_hash(k) & hi_mask) | id; });
}

// Heads of runs of >= 2 equal hashes; appended in any order through a warp-aggregated cursor.
__global__ void k_find_groups(const uint64_t* __restrict__ recs, int64_t V, int idbits, uint64_t* __restrict__ gstart,
                              uint32_t* __restrict__ gsize, unsigned long long* __restrict__ counter, int64_t cap) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool head = false;
    uint64_t k = 0;
    if (i < V) {
        k = recs[i] >> idbits;
        head = (i == 0 || (recs[i - 1] >> idbits) != k) && (i + 1 < V && (recs[i + 1] >> idbits) == k);
    }
    unsigned m = __ballot_sync(0xffffffffu, head);
    if (m == 0) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!head) return;
    unsigned long long slot = base + __popc(m & ((1u << lane) - 1u));
    int64_t j = i + 2;
    while (j < V && (recs[j] >> idbits) == k) j++;
    if ((int64_t)slot < cap) {
        gstart[slot] = (uint64_t)i;
        gsize[slot] = (uint32_t)(j - i);
    }
}

__global__ void k_pair_counts(const uint32_t* __restrict__ gsize, int64_t G, uint64_t* __restrict__ cnt) {
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    uint64_t s = gsize[g];
    cnt[g] = s * (s - 1) / 2;
}

constexpr int kEmitPer = 8;


__global__ void k_emit(const uint64_t* __restrict__ recs, const uint64_t* __restrict__ gstart,
                       const uint32_t* __restrict__ gsize, const uint64_t* __restrict__ goff, int64_t G, uint64_t P,
                       int idbits, uint64_t* __restrict__ pairs) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t p = t * kEmitPer;
    if (p >= P) return;
    uint64_t pend = p + kEmitPer < P ? p + kEmitPer : P;
    int64_t lo = 0, hi = G - 1;
    while (lo < hi) {
        int64_t mid = (lo + hi + 1) >> 1;
        if (goff[mid] <= p) lo = mid;
        else hi = mid - 1;
    }
    int64_t g = lo;
    uint64_t s = gsize[g];
    uint64_t base = gstart[g];
    uint64_t l = p - goff[g];
    double b2 = (double)(2 * s - 1);
    int64_t ii = (int64_t)floor((b2 - sqrt(b2 * b2 - 8.0 * (double)l)) * 0.5);
    if (ii < 0) ii = 0;
    uint64_t i = (uint64_t)ii;
    while (i + 1 < s && tri_row_start(i + 1, s) <= l) i++;
    while (i > 0 && tri_row_start(i, s) > l) i--;
    uint64_t j = i + 1 + (l - tri_row_start(i, s));
    const uint64_t idmask = (1ull << idbits) - 1ull;
    for (; p < pend; p++) {
        uint64_t a = recs[base + i] & idmask, b = recs[base + j] & idmask;
        uint64_t x = a < b ? a : b, y = a < b ? b : a;
        pairs[p] = (x << idbits) | y;
        if (++j == s) {
            ++i;
            j = i + 1;
            if (i + 1 >= s) {
                if (++g >= G) break;
                s = gsize[g];
                base = gstart[g];
                i = 0;
                j = 1;
            }
        }
    }
}

// Distance of two full-length sequences as the reference reports it
// (S/src/kernel.cu:235-300,359-392); *keep says whether the pair is output.
__device__ int pair_distance(const uint8_t* a, int la, const uint8_t* b, int lb, int d, int measure, bool* keep) {
    if (measure == kHamming) {
        int raw;
        int dv = hamming_ref(a, la, b, lb, &raw);
        bool k = dv <= d;
        // a wrapped counter (lengths >= 128) can accept a far pair: the reference outputs it
        // only when it was a candidate, i.e. when the 18-residue prefixes share a variant
        if (k && raw > d) k = prefixes_share_variant(a, la, b, lb, d);
        *keep = k;
        return dv;
    }
    int diff = la > lb ? la - lb : lb - la;
    if (diff > d) {
        *keep = false;
        return diff;
    }
    int dv;
    if (la <= 32 && la <= lb) dv = lev_myers<uint32_t>(a, la, b, lb);
    else if (lb <= 32 && lb <= la) dv = lev_myers<uint32_t>(b, lb, a, la);
    else if (la <= 64 && la <= lb) dv = lev_myers64(a, la, b, lb);
    else if (lb <= 64) dv = lev_myers64(b, lb, a, la);
    else {
        int col[kMaxInputLength + 1];
        dv = lev_dp(a, la, b, lb, col, d);
    }
    *keep = dv <= d;
    return dv;
}

// ------------------------------------------------------------------ candidate dedup
// Most candidate pairs are repeats (a close pair shares many deletion variants). Before the
// pair sort they go through a hash set in HBM (open addressing, linear probing):
// the first insertion of a pair appends it to `uniq`; repeats and self pairs are dropped, so
// only distinct pairs are sorted and verified. A slot holds tag | pair, the tag being the
// search's epoch in the top kDedupTagBits bits; a slot with another epoch is free, so the table
// is cleared only when allocated and when the epoch wraps. Pairs must fit in kDedupKeyBits
// bits (2 * id_bits <= 48, n <= 2^24). Slot hash: the SplitMix64 finaliser (Steele, Lea and
// Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014). With uniq == nullptr
// the pairs are only inserted (the rebuild of a grown table from the distinct list).
// Partitions: a table larger than L2 makes every first insertion a DRAM access, so the table is
// cut into 2^part_bits regions of 2^k slots each, the top part_bits bits of a pair's slot hash
// choosing the region; one launch per region passes over all candidates and inserts those of
// its region, so the region it probes stays in L2.
constexpr int kDedupKeyBits = 48;
constexpr int kDedupTagBits = 64 - kDedupKeyBits;
constexpr uint64_t kDedupTagMask = ~((1ull << kDedupKeyBits) - 1ull);
constexpr int64_t kDedupMinPairs = int64_t(1) << 15;  // below this the plain sort is as fast
// An insertion that probes this many slots gives up and asks for a larger table (the table is
// sized from the previous search's share of distinct pairs, which may not hold for this one).
constexpr uint32_t kDedupMaxProbes = 256;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Each block takes kDedupPer * kThreads candidates per step (a thread's first probes are issued
// together) and reserves the step's distinct pairs in `uniq` with one atomic. With one atomic
// per warp, nearly every warp (about 95% at 10M, where one candidate in eleven is new) hit the
// single counter: on B200 the 10M search's 56.6M candidates took 1.76 ms that way and take
// 0.65 ms with one atomic per block and step. (Smaller tables, 2^24 and 2^23 slots instead of
// 2^25, measured slower in both forms: 0.69 and 0.90 ms here; longer probe runs cost more than
// the L2 hits save.)
constexpr int kDedupPer = 4;
constexpr int64_t kDedupStep = (int64_t)kThreads * kDedupPer;

__global__ void __launch_bounds__(kThreads) k_pair_dedup(const uint64_t* __restrict__ pairs, int64_t P, int idbits,
                                                         unsigned long long* __restrict__ table, uint64_t tmask,
                                                         uint64_t tag, uint64_t* __restrict__ uniq,
                                                         unsigned long long* __restrict__ n_uniq,
                                                         unsigned long long* __restrict__ n_full,
                                                         const unsigned long long* __restrict__ P_dev, int part_bits,
                                                         uint32_t part) {
    __shared__ uint32_t s_warp[kThreads / 32];
    __shared__ unsigned long long s_base;
    // P_dev (graph form): the count is read on the device (at most P) and the grid strides
    if (P_dev) P = (int64_t)min((unsigned long long)P, *P_dev);
    table += (size_t)part * (tmask + 1);  // this region
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint64_t idmask = (1ull << idbits) - 1ull;
    const int64_t stride = (int64_t)gridDim.x * kDedupStep;
    for (int64_t b0 = (int64_t)blockIdx.x * kDedupStep; b0 < P; b0 += stride) {  // the same steps for the whole block
        uint64_t p[kDedupPer], h[kDedupPer];
        unsigned long long v[kDedupPer];
        bool live[kDedupPer], fresh[kDedupPer];
#pragma unroll
        for (int k = 0; k < kDedupPer; k++) {
            const int64_t i = b0 + (int64_t)k * kThreads + threadIdx.x;
            p[k] = 0;
            h[k] = 0;
            live[k] = fresh[k] = false;
            if (i < P) {
                p[k] = __ldcs(pairs + i);  // read once: evict-first, so that the table's lines stay in L2
                const uint64_t hm = mix64(p[k]);
                live[k] = (p[k] >> idbits) != (p[k] & idmask) &&
                          (part_bits == 0 || (uint32_t)(hm >> (64 - part_bits)) == part);
                h[k] = hm & tmask;
            }
        }
#pragma unroll
        for (int k = 0; k < kDedupPer; k++) v[k] = live[k] ? ld_relaxed_u64(table + h[k]) : 0ull;
#pragma unroll
        for (int k = 0; k < kDedupPer; k++) {
            if (!live[k]) continue;
            const unsigned long long want = tag | p[k];
            uint64_t hh = h[k];
            unsigned long long vv = v[k];
            for (uint32_t probes = 0;;) {
                if ((vv & kDedupTagMask) != tag) {  // free in this search
                    const unsigned long long old = atomicCAS(table + hh, vv, want);
                    if (old == vv) {
                        fresh[k] = true;
                        break;
                    }
                    vv = old;  // taken meanwhile: it now holds a pair of this search
                    continue;
                }
                if (vv == want) break;  // a repeat
                hh = (hh + 1) & tmask;
                if (++probes > kDedupMaxProbes) {  // table too full: the host reruns with a larger one
                    atomicAdd(n_full, 1ull);
                    break;
                }
                vv = ld_relaxed_u64(table + hh);
            }
        }
        if (uniq == nullptr) continue;  // (uniform over the block)
        unsigned mask[kDedupPer];
        uint32_t mine = 0;
#pragma unroll
        for (int k = 0; k < kDedupPer; k++) {
            mask[k] = __ballot_sync(0xffffffffu, fresh[k]);
            mine += __popc(mask[k]);
        }
        if (lane == 0) s_warp[warp] = mine;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
#pragma unroll
            for (int w = 0; w < kThreads / 32; w++) t += s_warp[w];
            s_base = t ? atomicAdd(n_uniq, (unsigned long long)t) : 0ull;
        }
        __syncthreads();
        unsigned long long base = s_base;
        for (unsigned w = 0; w < warp; w++) base += s_warp[w];
        const unsigned lt = (1u << lane) - 1u;
#pragma unroll
        for (int k = 0; k < kDedupPer; k++) {
            if (fresh[k]) uniq[base + __popc(mask[k] & lt)] = p[k];
            base += __popc(mask[k]);
        }
        __syncthreads();  // s_warp and s_base are rewritten by the next step
    }
}

// Table regions: each at most kDedupRegionBytes. Regions of 64 MiB (a quarter of the 10M
// workload's 256 MiB table, so that each pass's probes stay in L2) were measured slower on B200
// (2.97 ms against 1.75 ms for 56M candidates: four passes over the candidates cost more than
// the L2 hits save), so tables up to 1 GiB take one pass.
constexpr uint64_t kDedupRegionBytes = uint64_t(1) << 30;

static int dedup_part_bits(uint64_t T) {
    int pb = 0;
    while ((T >> pb) * sizeof(uint64_t) > kDedupRegionBytes && (T >> pb) > 1024) pb++;
    return pb;
}

// One pass per table region over the P candidates (grid-stride with `grid` blocks when P_dev
// gives the count on the device).
static void launch_pair_dedup(const uint64_t* pairs, int64_t P, int idbits, unsigned long long* table, uint64_t T,
                              uint64_t tag, uint64_t* uniq, unsigned long long* n_uniq, unsigned long long* n_full,
                              const unsigned long long* P_dev, unsigned grid, cudaStream_t s) {
    const int pb = dedup_part_bits(T);
    const uint64_t region = T >> pb;
    // `grid` bounds the blocks; one step of kDedupStep candidates per block needs no more
    grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)grid, (P + kDedupStep - 1) / kDedupStep));
    for (uint32_t part = 0; part < (1u << pb); part++)
        XTN_LAUNCH("pair_dedup", k_pair_dedup<<<grid, kThreads, 0, s>>>(pairs, P, idbits, table, region - 1, tag, uniq,
                                                                        n_uniq, n_full, P_dev, pb, part));
}

// Verification of the sorted candidate pairs. Only the first of each run of equal pairs, with
// x != y, is verified; the others get distance 0 and are not kept. Most candidates are repeats
// (a close pair shares many deletion variants), so each warp takes kVerifyPer * 32 consecutive
// candidates, lists the ones to verify in shared memory and spreads them over its lanes.
// The verification variant (context option verify_per, chosen by the autotuner) is the number
// of candidates per lane a warp lists before verifying: more amortises the listing over repeats
// of sorted candidates, fewer keeps the lanes busier when the candidates are distinct already.
constexpr int kVerifyPer = 4;
constexpr int kVerifyWarps = kThreads / 32;

template <int PER>
__global__ void __launch_bounds__(kThreads) k_verify_t(const uint64_t* __restrict__ pairs, int64_t P, int idbits,
                                                       const uint8_t* __restrict__ chars, const uint32_t* __restrict__ offs,
                                                       const int32_t* __restrict__ rows, int d, int measure,
                                                       int8_t* __restrict__ dist, uint8_t* __restrict__ flag,
                                                       const unsigned long long* __restrict__ P_dev) {
    static_assert(PER >= 1 && PER <= 8, "slots are 8-bit");
    __shared__ uint64_t s_pair[kVerifyWarps][32 * PER];
    __shared__ uint8_t s_slot[kVerifyWarps][32 * PER];
    if (P_dev) P = (int64_t)min((unsigned long long)P, *P_dev);  // graph form: grid sized for P at most
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = ((int64_t)blockIdx.x * kVerifyWarps + warp) * (32 * PER);
    if (base >= P) return;  // whole warp
    const uint64_t idmask = (1ull << idbits) - 1ull;
    const unsigned lt = (1u << lane) - 1u;
    uint64_t carry = base > 0 ? pairs[base - 1] : 0ull;  // the candidate before each row's lane 0
    uint32_t n_work = 0;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        const int64_t i = base + k * 32 + lane;
        const bool in = i < P;
        const uint64_t p = in ? pairs[i] : 0ull;
        uint64_t prev = __shfl_up_sync(0xffffffffu, p, 1);
        if (lane == 0) prev = carry;
        carry = __shfl_sync(0xffffffffu, p, 31);
        const bool need = in && (i == 0 || prev != p) && (p >> idbits) != (p & idmask);
        const unsigned mask = __ballot_sync(0xffffffffu, need);
        if (need) {
            const uint32_t w = n_work + __popc(mask & lt);
            s_pair[warp][w] = p;
            s_slot[warp][w] = (uint8_t)(k * 32 + lane);
        } else if (in) {
            dist[i] = 0;
            flag[i] = 0;
        }
        n_work += __popc(mask);
    }
    __syncwarp();
    for (uint32_t w = lane; w < n_work; w += 32) {
        const uint64_t p = s_pair[warp][w];
        const int64_t i = base + s_slot[warp][w];
        const uint32_t x = (uint32_t)(p >> idbits), y = (uint32_t)(p & idmask);
        const int rx = rows ? rows[x] : (int)x, ry = rows ? rows[y] : (int)y;
        const uint32_t sa = offs[rx], sb = offs[ry];
        bool keep = false;
        const int dv = pair_distance(chars + sa, (int)(offs[rx + 1] - sa), chars + sb, (int)(offs[ry + 1] - sb), d,
                                     measure, &keep);
        dist[i] = (int8_t)dv;
        flag[i] = keep ? 1 : 0;
    }
}

__global__ void k_compact(const uint64_t* __restrict__ pairs, int64_t P, int idbits, const int8_t* __restrict__ dist,
                          const uint8_t* __restrict__ flag, const uint32_t* __restrict__ pos, xtn_int2* __restrict__ out,
                          int8_t* __restrict__ out_dist, const unsigned long long* __restrict__ P_dev) {
    if (P_dev) P = (int64_t)min((unsigned long long)P, *P_dev);
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P || !flag[i]) return;
    uint64_t p = pairs[i];
    uint32_t o = pos[i];
    out[o] = xtn_int2{(int32_t)(p >> idbits), (int32_t)(p & ((1ull << idbits) - 1ull))};
    out_dist[o] = dist[i];
}

// ------------------------------------------------------------------ device buffers
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};

static int ensure(DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.cap >= bytes) return XTN_SUCCESS;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t nb = bytes + bytes / 8;
    nb = (nb + 255) & ~size_t(255);
    cudaError_t e = cudaMalloc(&b.p, nb);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        set_err(std::string("device allocation of ") + std::to_string(nb) + " bytes failed: " + cudaGetErrorString(e));
        return XTN_ERR_NOMEM;
    }
    b.cap = nb;
    return XTN_SUCCESS;
}

static void release(DevBuf& b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
}

template <typename T>
static T* P(DevBuf& b) {
    return reinterpret_cast<T*>(b.p);
}

static inline unsigned blocks_for(int64_t n, int per_block = kThreads) {
    int64_t b = (n + per_block - 1) / per_block;
    return (unsigned)(b > 0 ? b : 1);
}

static int id_bits_for(int64_t n) {
    int b = 1;
    while ((int64_t(1) << b) < n) b++;
    return b;
}

// Launches the verification variant `per` (1, 4 or 8) over capacity P (device count P_dev).
static void launch_verify(int per, const uint64_t* pairs, int64_t P, int idbits, const uint8_t* chars,
                          const uint32_t* offs, const int32_t* rows, int d, int measure, int8_t* dist, uint8_t* flag,
                          const unsigned long long* P_dev, cudaStream_t s) {
    if (per == 1)
        XTN_LAUNCH("verify", k_verify_t<1><<<blocks_for(P, kThreads * 1), kThreads, 0, s>>>(
                                 pairs, P, idbits, chars, offs, rows, d, measure, dist, flag, P_dev));
    else if (per == 8)
        XTN_LAUNCH("verify", k_verify_t<8><<<blocks_for(P, kThreads * 8), kThreads, 0, s>>>(
                                 pairs, P, idbits, chars, offs, rows, d, measure, dist, flag, P_dev));
    else
        XTN_LAUNCH("verify", k_verify_t<kVerifyPer><<<blocks_for(P, kThreads * kVerifyPer), kThreads, 0, s>>>(
                                 pairs, P, idbits, chars, offs, rows, d, measure, dist, flag, P_dev));
}


}  // namespace xtn

using namespace xtn;

enum { S_PACK, S_GEN, S_KSORT, S_GROUP, S_EMIT, S_PSORT, S_VERIFY, S_OUT, S_COUNT };

struct xtn_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[S_COUNT + 1] = {};
    // inputs (host-buffer API)
    DevBuf chars, offs, info, lencheck;
    // pipeline
    DevBuf keys, klen, vcnt, voff, recA, recB, gstart, gsize, gcnt, goff, pairA, pairB, dist, flag, fpos;
    DevBuf scratch64, scratch32, counter;
    DevBuf os_scratch, os_status, dev_err;  // single-sweep sort scratch, status words, wait-error count
    DevBuf scan_status;      // single-pass scan status words
    uint32_t os_epoch = 0;
    DevBuf dd_table;         // candidate-pair hash set (tag | pair per slot)
    uint32_t dd_epoch = 0;
    double dd_share = 1.0;   // distinct share of the previous search's candidates (table sizing)
    int dedup_slots_log2 = 0;  // > 0: the one-round hash set's first table has 2^this slots
    int pair_dedup = 1;      // candidate pairs through the hash set before the pair sort (2: table always sized by share)
    DevBuf bcounts, boffs, btotals, bstart, bdesc, bjobs, bfall, bcnt, fbA, fbB, runinfo, tcnt, toff, ktab, tseq;
    int sms = 148;
    int engine = 0;         // 0: hash buckets, 1: full radix sort of the records
    int onesweep = 1;       // radix sorts by single-sweep passes (0: classic passes)
    bool attrs_set = false;
    int bucket_bits_max = kMaxFirstLevelBits;
    int scatter_ctas_per_sm = 0;  // 0: as many as the stage shape's shared memory allows
    int group_tma = 1;
    int key_tables = 1;     // d <= 2 variant hashes from per-sequence tables
    int verify_per = 1;     // verification variant: candidates listed per lane (1, 4, 8)
    int group_persistent = 1;  // grouping by persistent CTAs on a descriptor queue (large grids)
    int shard_count = 1, shard_index = 0;  // this search covers shard shard_index of shard_count
    int flat_gen = 1;       // one-round first level: generate in sequence order, then partition
    int split_fill = 87;    // split sub-buckets sized at this percentage of group_cap
    int split_slotted = 1;  // one-round searches split in one pass into fixed slots
    uint32_t wait_polls = kScanPollLimit;  // bound on a single-pass scan's look-back polls
    int wait_fault_test = 0;  // 1: the next variant-offset scan withholds tile 0's status word
    int stage_chunk = 4096;  // records per staged chunk of the first-level scatter (2048 | 4096 | 8192)
    int split_chunk = 0;     // the same for the split (2048 | 4096 | 8192; 0: by bucket size)
    int split_slices = kSplitSlices;  // CTAs (one cluster) per split bucket: 1 | kSplitSlices
    uint32_t group_cap = kGroupCap;
    double last_pc_per_rec = 0;  // candidates per variant record of the previous run (buffer sizing)
    // rounds: memory model and the second stream of the multi-round loop
    int64_t memory_budget = 0;      // bytes a search may hold on the device; 0: 80% of what is free
    int64_t max_round_records = 0;  // records per round at most; 0: from the budget
    int round_overlap = 1;          // 1: a round's pair dedup runs on stream2 during the next round
    size_t total_mem = 0;           // device memory size
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_round[2] = {};
    DevBuf pairA2, ddcnt;
    DevBuf scur;             // sub-bucket cursors of the slotted split
    DevBuf gruns;            // shard exchange: runs gathered into contiguous first-level buckets
    // graph form of the device-resident search (option "graph")
    int graph_mode = 0;
    void* graph = nullptr;  // GraphState (below)
    void* ograph = nullptr; // OverlapGraph (below)
    // autotuner: shapes chosen per input class (see TuneKey), and whether device-resident
    // searches consult (and fill) that cache by themselves
    int autotune_auto = 0;
    void* tune_cache = nullptr;
    // results
    DevBuf out_pairs, out_dist, out_freq;
    uint64_t* h_scalar = nullptr;  // pinned
    void* h_stage = nullptr;       // pinned output staging
    size_t h_stage_cap = 0;
    int64_t n_out = 0;
    bool overlap_result = false;
    xtn_stats stats{};
    void* overlap_bufs = nullptr;
    KernelProfiler prof;
    std::vector<std::string> kt_names;
    std::vector<double> kt_ms;
    std::vector<int64_t> kt_launches;
};

namespace xtn {

static int read_scalar(xtn_context* c, const void* dptr, size_t bytes, uint64_t* out) {
    *c->h_scalar = 0;
    XTN_CK(cudaMemcpyAsync(c->h_scalar, dptr, bytes, cudaMemcpyDeviceToHost, c->stream));
    XTN_CK(cudaStreamSynchronize(c->stream));
    *out = *c->h_scalar;
    return XTN_SUCCESS;
}

// Length check of device-resident offsets (k_check_lengths) into c->lencheck; the caller reads
// the word with its next synchronisation and passes it to length_check_result.
static int launch_length_check(xtn_context* c, const uint32_t* offs, const int32_t* rows, int n) {
    XTN_TRY(ensure(c->lencheck, 16));
    XTN_CK(cudaMemsetAsync(c->lencheck.p, 0xff, 4, c->stream));
    XTN_LAUNCH("check_lengths", k_check_lengths<<<blocks_for(n), kThreads, 0, c->stream>>>(
                                    offs, rows, n, P<unsigned int>(c->lencheck)));
    XTN_CK(cudaGetLastError());
    return XTN_SUCCESS;
}

static int length_check_result(xtn_context* c, uint32_t first_bad) {
    (void)c;
    if (first_bad == 0xffffffffu) return XTN_SUCCESS;
    set_err("sequence " + std::to_string(first_bad) + " has an invalid length");
    return XTN_ERR_ARG;
}

static void begin_run(xtn_context* c) {
    c->prof.reset(c->stream);
    current_profiler() = &c->prof;
}

// After the stream has drained: per-kernel totals (profiling on) and the launch count.
static void end_run(xtn_context* c) {
    current_profiler() = nullptr;
    c->stats.n_launches = c->prof.launches;
    c->kt_names.clear();
    c->kt_ms.clear();
    c->kt_launches.clear();
    if (!c->prof.on) return;
    cudaStreamSynchronize(c->stream);
    for (size_t i = 0; i < c->prof.used; i++) {
        const KernelProfiler::Rec& r = c->prof.recs[i];
        float ms = 0;
        cudaEventElapsedTime(&ms, r.a, r.b);
        size_t k = 0;
        while (k < c->kt_names.size() && c->kt_names[k] != r.name) k++;
        if (k == c->kt_names.size()) {
            c->kt_names.push_back(r.name);
            c->kt_ms.push_back(0);
            c->kt_launches.push_back(0);
        }
        c->kt_ms[k] += ms;
        c->kt_launches[k]++;
    }
}

static int ensure_err_word(xtn_context* c);

// Single-pass scans (scan_exclusive_1p); their status words live in c->scan_status and a wait
// that reaches its bound is counted in c->dev_err, which each entry point checks at its end.
// withhold_tile0: the fault test of the bounded waits (context option "wait_fault_test"); only
// the variant-offset scan takes it, whose result the host checks before anything consumes it.
template <typename In, typename Out>
static int scan_1p(xtn_context* c, const In* in, Out* out, int64_t n, int withhold_tile0 = 0) {
    XTN_TRY(ensure(c->scan_status, sizeof(unsigned long long) * scan_1p_words(n)));
    XTN_TRY(ensure_err_word(c));
    scan_exclusive_1p<In, Out>(in, out, n, P<unsigned long long>(c->scan_status), P<unsigned int>(c->dev_err),
                               c->stream, c->wait_polls, withhold_tile0);
    return XTN_SUCCESS;
}

static int scan_u32_to_u64(xtn_context* c, const uint32_t* in, uint64_t* out, int64_t n) {
    return scan_1p<uint32_t, uint64_t>(c, in, out, n);
}

static int scan_u64(xtn_context* c, const uint64_t* in, uint64_t* out, int64_t n) {
    return scan_1p<uint64_t, uint64_t>(c, in, out, n);
}

// Kernel names of one sort (classic passes or single-sweep passes).
struct SortNames {
    const char* up;
    const char* down;
    const char* hist;
    const char* pass;
};
#define XTN_SORT_NAMES(p) (SortNames{p "_upsweep", p "_downsweep", p "_hist", p "_pass"})

// Single-sweep passes are used up to this many keys. They save the classic passes' count
// kernels, scans and launches, which dominate small sorts. Above it the classic passes were
// measured faster on B200 (55M candidate pairs: 2.6 ms against 3.2 ms), because each tile's
// look-back latency is exposed at five CTAs per SM.
constexpr int64_t kOsMaxKeys = int64_t(1) << 24;

static int ensure_err_word(xtn_context* c) {
    if (c->dev_err.p) return XTN_SUCCESS;
    XTN_TRY(ensure(c->dev_err, 16));
    XTN_CK(cudaMemsetAsync(c->dev_err.p, 0, 16, c->stream));
    return XTN_SUCCESS;
}

// Sorts n keys by bits [lo, hi): single-sweep passes (look-back) up to kOsMaxKeys keys, else
// the classic count / scan / scatter passes.
static int sort_u64(xtn_context* c, DevBuf& a, DevBuf& b, int64_t n, int lo, int hi, uint64_t** result,
                    SortNames names) {
    const int passes = (hi - lo + kRadixBits - 1) / kRadixBits;
    const int64_t words = onesweep_status_words(n);
    if (c->onesweep && n <= kOsMaxKeys && passes <= kOsMaxPasses) {
        XTN_TRY(ensure(c->os_scratch, sizeof(uint32_t) * kOsScratchWords));
        XTN_TRY(ensure_err_word(c));
        if (c->os_status.cap < sizeof(unsigned long long) * (size_t)words) {
            XTN_TRY(ensure(c->os_status, sizeof(unsigned long long) * (size_t)words));
            XTN_CK(cudaMemsetAsync(c->os_status.p, 0, c->os_status.cap, c->stream));
        }
        *result = onesweep_sort_u64(P<uint64_t>(a), P<uint64_t>(b), n, lo, hi, P<uint32_t>(c->os_scratch),
                                    P<unsigned long long>(c->os_status), (int64_t)(c->os_status.cap / 8), &c->os_epoch,
                                    P<unsigned int>(c->dev_err), c->sms, c->stream, names.hist, names.pass);
        return XTN_SUCCESS;
    }
    XTN_TRY(ensure(c->scratch32, sizeof(uint32_t) * radix_scratch_elems(n)));
    *result = radix_sort_u64(P<uint64_t>(a), P<uint64_t>(b), n, lo, hi, P<uint32_t>(c->scratch32), c->stream, names.up,
                             names.down);
    return XTN_SUCCESS;
}

// Reads (after the stream has drained up to here) and clears the count of device waits that
// gave up; nonzero means a result computed since the last check is unreliable.
static int check_err_word(xtn_context* c) {
    if (!c->dev_err.p) return XTN_SUCCESS;
    uint64_t e = 0;
    XTN_TRY(read_scalar(c, c->dev_err.p, 4, &e));
    if (e != 0) {
        XTN_CK(cudaMemsetAsync(c->dev_err.p, 0, 16, c->stream));
        set_err(std::to_string(e) + " look-back waits (radix sort or scan) did not complete in time");
        return XTN_ERR_CUDA;
    }
    return XTN_SUCCESS;
}

// Grows a buffer keeping its first `used` bytes.
static int ensure_keep(xtn_context* c, DevBuf& b, size_t bytes, size_t used) {
    if (b.cap >= bytes) return XTN_SUCCESS;
    DevBuf nb;
    XTN_TRY(ensure(nb, bytes));
    if (used) XTN_CK(cudaMemcpyAsync(nb.p, b.p, used, cudaMemcpyDeviceToDevice, c->stream));
    XTN_CK(cudaStreamSynchronize(c->stream));
    release(b);
    b = nb;
    return XTN_SUCCESS;
}

// Records of the fallback buckets desc[0..gridDim.x) copied one after another into `out`
// (bucket k at off[k]); one CTA per bucket.
__global__ void k_fallback_gather(const BucketDesc* __restrict__ desc, const uint64_t* __restrict__ off,
                                  const uint64_t* __restrict__ recA, const uint64_t* __restrict__ recB,
                                  uint64_t* __restrict__ out) {
    const BucketDesc f = desc[blockIdx.x];
    const uint64_t* src = (f.src ? recB : recA) + f.start;
    uint64_t* dst = out + off[blockIdx.x];
    for (uint32_t i = threadIdx.x; i < f.size; i += blockDim.x) dst[i] = src[i];
}

// Records gathered per batch of fallback buckets (more when one bucket alone is larger).
constexpr uint64_t kFallbackBatchRecords = uint64_t(1) << 26;

// Candidate pairs of a record array sorted by hash: runs of equal hash, every id pair of every
// run appended to `out` at index `base`. *count receives the number appended.
static int group_sorted(xtn_context* c, const uint64_t* recs, int64_t V, int idbits, DevBuf& out, uint64_t base,
                        uint64_t* count) {
    cudaStream_t s = c->stream;
    XTN_TRY(ensure(c->counter, 64));
    int64_t gcap = std::max<int64_t>(1 << 16, V / 8);
    uint64_t G = 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        XTN_TRY(ensure(c->gstart, sizeof(uint64_t) * gcap));
        XTN_TRY(ensure(c->gsize, sizeof(uint32_t) * gcap));
        XTN_CK(cudaMemsetAsync(c->counter.p, 0, 8, s));
        XTN_LAUNCH("find_groups", k_find_groups<<<blocks_for(V), kThreads, 0, s>>>(
                                      recs, V, idbits, P<uint64_t>(c->gstart), P<uint32_t>(c->gsize),
                                      P<unsigned long long>(c->counter), gcap));
        XTN_CK(cudaGetLastError());
        XTN_TRY(read_scalar(c, c->counter.p, 8, &G));
        if ((int64_t)G <= gcap) break;
        gcap = (int64_t)G;
    }
    c->stats.n_groups += (int64_t)G;
    *count = 0;
    if (G == 0) return XTN_SUCCESS;
    XTN_TRY(ensure(c->gcnt, sizeof(uint64_t) * (G + 1)));
    XTN_TRY(ensure(c->goff, sizeof(uint64_t) * (G + 1)));
    XTN_LAUNCH("pair_counts", k_pair_counts<<<blocks_for((int64_t)G), kThreads, 0, s>>>(P<uint32_t>(c->gsize),
                                                                                       (int64_t)G, P<uint64_t>(c->gcnt)));
    XTN_CK(cudaGetLastError());
    XTN_TRY(scan_u64(c, P<uint64_t>(c->gcnt), P<uint64_t>(c->goff), (int64_t)G));
    uint64_t Pc = 0;
    XTN_TRY(read_scalar(c, P<uint64_t>(c->goff) + G, 8, &Pc));
    if (Pc == 0) return XTN_SUCCESS;
    XTN_TRY(ensure_keep(c, out, sizeof(uint64_t) * (base + Pc) + 64, sizeof(uint64_t) * base));
    uint64_t threads = (Pc + kEmitPer - 1) / kEmitPer;
    XTN_LAUNCH("emit", k_emit<<<blocks_for((int64_t)threads), kThreads, 0, s>>>(
                           recs, P<uint64_t>(c->gstart), P<uint32_t>(c->gsize), P<uint64_t>(c->goff), (int64_t)G, Pc,
                           idbits, P<uint64_t>(out) + base));
    XTN_CK(cudaGetLastError());
    *count = Pc;
    return XTN_SUCCESS;
}

// Sort engine: every record materialised in sequence order, radix-sorted by hash, grouped.
static int candidates_sorted(xtn_context* c, int n, int d, int idbits, uint64_t V, uint64_t* Pc) {
    cudaStream_t s = c->stream;
    XTN_TRY(ensure(c->recA, sizeof(uint64_t) * V + 64));
    XTN_TRY(ensure(c->recB, sizeof(uint64_t) * V + 64));
    XTN_LAUNCH("gen", k_gen<<<blocks_for(n), kThreads, 0, s>>>(
                          P<u128>(c->keys), P<uint8_t>(c->klen), P<uint64_t>(c->runinfo),
                          d <= 2 && c->key_tables ? P<uint64_t>(c->ktab) : nullptr, P<uint64_t>(c->voff), n, d, idbits,
                          P<uint64_t>(c->recA)));
    XTN_CK(cudaGetLastError());
    XTN_CK(cudaEventRecord(c->ev[2], s));
    uint64_t* recs = nullptr;
    XTN_TRY(sort_u64(c, c->recA, c->recB, (int64_t)V, idbits, 64, &recs, XTN_SORT_NAMES("key_sort")));
    XTN_CK(cudaEventRecord(c->ev[3], s));
    XTN_TRY(group_sorted(c, recs, (int64_t)V, idbits, c->pairA, 0, Pc));
    XTN_CK(cudaEventRecord(c->ev[4], s));
    return XTN_SUCCESS;
}

// Bucket engine (xtn_bucket.cuh). A search's first-level plan (bucket bits, tiles, per-tile
// bucket counts, bucket starts, the d = 2 task map) is made once; the records are then
// produced, split and grouped in one or more rounds, each over a contiguous range of
// first-level buckets (bucket_round).
struct BucketPlan {
    int b1 = 1, nb = 2, ntiles = 1, tile = 1;
    bool small = false, staged = false;
    bool flat = false;  // generate in sequence order (recB), then partition (k_bucket_gen / k_bucket_partition)
    bool slotted = false;  // one-pass split into fixed slots (k_bucket_split_slotted)
    uint64_t sub_bound = 0;  // slotted: sub-buckets of all jobs, at most
    uint64_t recb = 0;       // records buffer B must hold
    const uint32_t* tseq = nullptr;
};

__global__ void k_set_u64(unsigned long long* p, unsigned long long v) { *p = v; }

static int bucket_attrs(xtn_context* c) {
    if (c->attrs_set) return XTN_SUCCESS;
    XTN_CK(cudaFuncSetAttribute(k_bucket_count, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    XTN_CK(cudaFuncSetAttribute(k_bucket_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    XTN_CK(cudaFuncSetAttribute(k_bucket_scatter_staged<StageLarge>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(ScatterSmem<StageLarge>)));
    XTN_CK(cudaFuncSetAttribute(k_bucket_scatter_staged<StageSmall>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(ScatterSmem<StageSmall>)));
    XTN_CK(cudaFuncSetAttribute(k_bucket_scatter_staged<StageHuge>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(ScatterSmem<StageHuge>)));
    XTN_CK(cudaFuncSetAttribute(k_bucket_split_staged<StageLarge, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(StageSmem<StageLarge>)));
    XTN_CK(cudaFuncSetAttribute(k_bucket_split_staged<StageLarge, kSplitSlices>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(StageSmem<StageLarge>)));
    XTN_CK(cudaFuncSetAttribute(k_bucket_split_staged<SplitSmall, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(StageSmem<SplitSmall>)));
    XTN_CK(cudaFuncSetAttribute(k_bucket_split_staged<SplitSmall, kSplitSlices>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(StageSmem<SplitSmall>)));
    XTN_CK(cudaFuncSetAttribute(k_bucket_group<GroupLarge>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(GroupSmem<GroupLarge>)));
    XTN_CK(cudaFuncSetAttribute(k_bucket_group<GroupSmall>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(GroupSmem<GroupSmall>)));
    XTN_CK(cudaFuncSetAttribute(k_bucket_partition<StageHuge>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(StageSmem<StageHuge>)));
    XTN_CK(cudaFuncSetAttribute(k_bucket_split_slotted<StageLarge, kSplitSlices>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(StageSmem<StageLarge>)));
    XTN_CK(cudaFuncSetAttribute(k_bucket_split_slotted<StageHuge, kSplitSlices>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(StageSmem<StageHuge>)));
    c->attrs_set = true;
    return XTN_SUCCESS;
}

// The grouping kernel in the shape group_cap asks for: one CTA per descriptor (ndesc of them),
// or persistent CTAs (MIN_CTAS per SM) reading the descriptor count on the device.
static int launch_group(xtn_context* c, uint32_t ndesc, bool persistent, int idbits, uint64_t* pairs, uint64_t cap,
                        uint32_t desc_cap, cudaStream_t s) {
#define XTN_GROUP(G)                                                                                              \
    XTN_LAUNCH("bucket_group",                                                                                   \
               k_bucket_group<G><<<persistent ? (unsigned)c->sms * G::kMinCtas : ndesc, G::kThreads,             \
                                   sizeof(GroupSmem<G>), s>>>(                                                   \
                   P<BucketDesc>(c->bdesc), P<uint64_t>(c->recA), P<uint64_t>(c->recB), idbits, pairs, cap,     \
                   P<unsigned long long>(c->counter), P<unsigned int>(c->counter) + 2, c->group_tma,           \
                   P<BucketDesc>(c->bfall), desc_cap, P<unsigned int>(c->bcnt),                                 \
                   persistent ? P<unsigned int>(c->bcnt) + kCntDesc : nullptr))
    if (persistent) XTN_CK(cudaMemsetAsync(P<unsigned int>(c->bcnt) + kCntNext, 0, sizeof(unsigned int), s));
    if (c->group_cap <= (uint32_t)kGroupSmallCap) XTN_GROUP(GroupSmall);
    else XTN_GROUP(GroupLarge);
#undef XTN_GROUP
    XTN_CK(cudaGetLastError());
    return XTN_SUCCESS;
}

// Largest first-level bucket bits: the staged scatter's fan-out bounds it for d <= 2 with key
// tables; the direct scatter (d > 2, or per-key hashing) takes up to 2^14 buckets, which keeps
// the buckets of very large variant counts (10M sequences at d = 3: ~6e9) small enough for the
// split to bring them to shared-memory size.
constexpr int kDirectBucketBitsMax = 14;
constexpr uint64_t kFirstLevelRecords = 1500000;
constexpr uint64_t kFirstLevelRecordsFlat = 2500000;

// The first-level plan: count pass over every variant (per-tile histograms of the top b1 hash
// bits), per-tile offsets inside each bucket, bucket starts (c->bstart, nb + 1 entries) and, for
// the staged scatter at d = 2, the balanced task map.
// The first-level shape for n sequences and V variant records (no device work).
// Sub-buckets at most and records of buffer B for the split of V records in b_n first-level
// buckets: with the slotted split, ceil(size / target) sub-buckets per split bucket and a slot of
// group_cap records each.
static void slot_sizes(const xtn_context* c, const BucketPlan& bp, uint64_t V, uint32_t b_n, uint64_t* sub_bound,
                       uint64_t* recb) {
    const uint64_t sub_target = std::max<uint64_t>(1, (uint64_t)c->group_cap * c->split_fill / 100);
    *sub_bound = V / sub_target + (uint64_t)b_n + 1;
    *recb = bp.slotted ? std::max<uint64_t>(V, *sub_bound * c->group_cap) : V;
}

// one_round: every record is kept at once, so the two-pass first level (option flat_gen) can
// run; bp->flat says whether it does.
static void bucket_shape(const xtn_context* c, int n, int d, uint64_t V, BucketPlan* bp, bool one_round) {
    const bool small = c->stage_chunk == 2048;
    const bool tables = d <= 2 && c->key_tables;
    const bool flat = one_round && c->flat_gen && tables && c->stage_chunk == 4096;
    // the staged scatter's fan-out bounds the first-level bits; the direct scatter (d > 2, or
    // per-key hashing) takes up to 2^14 buckets
    const int fan_bits = tables ? (small ? 9 : 10) : kDirectBucketBitsMax;
    const int lim = tables ? std::min(c->bucket_bits_max, fan_bits) : std::max(c->bucket_bits_max, kDirectBucketBitsMax);
    int b1 = 1;
    // buckets of about 7000 records or more (up to 512 of them with the key tables)
    while (b1 < (tables ? std::min(lim, 9) : lim) && (V >> b1) > 7000) b1++;
    // first-level buckets of more than kFirstLevelRecords records make the split re-read its
    // slices from DRAM (a cluster's bucket no longer stays in L2) and write short runs: at 10M
    // sequences 1024 buckets instead of 512 cut the split from 10.5 to 7.5 ms for 1.7 ms more
    // one-pass scatter; at 1M, 512 stay faster. The two-pass first level's partition gains more
    // from the longer runs of 512 buckets (10M: partition 5.09 against 6.78 ms, split 7.94
    // against 6.66 ms), so it keeps buckets of up to kFirstLevelRecordsFlat records.
    while (b1 < lim && (V >> b1) > (flat ? kFirstLevelRecordsFlat : kFirstLevelRecords)) b1++;
    // enough buckets that the split (at most 2^kMaxSplitBits ways) can bring each to the
    // grouping capacity (the small grouping shape at 10M sequences needs 1024 of them)
    const uint64_t target = std::max<uint64_t>(1, (uint64_t)c->group_cap * 7 / 8);
    while (b1 < lim && ((V >> b1) >> kMaxSplitBits) > target) b1++;
    const int nb = 1 << b1;
    const int per_sm = c->scatter_ctas_per_sm ? c->scatter_ctas_per_sm  // count/scatter tiles per SM
                       : small                  ? ctas_per_sm_for<ScatterSmem<StageSmall>>()
                       : c->stage_chunk == 8192 ? ctas_per_sm_for<ScatterSmem<StageHuge>>()
                                                : ctas_per_sm_for<ScatterSmem<StageLarge>>();
    const int64_t wave = (int64_t)c->sms * per_sm;
    const int ntiles = (int)(wave * std::max<int64_t>(1, ((int64_t)n + wave * 4096 - 1) / (wave * 4096)));
    bp->b1 = b1;
    bp->nb = nb;
    bp->ntiles = ntiles;
    bp->tile = (n + ntiles - 1) / ntiles;
    bp->small = small;
    bp->staged = tables && b1 <= fan_bits;
    bp->flat = flat && bp->staged;
    // the slotted split: buffer B then holds a slot of group_cap records per sub-bucket, about
    // 1 / split_fill of the records plus one slot per first-level bucket (sized per round)
    bp->slotted = c->split_slotted != 0;
    slot_sizes(c, *bp, V, (uint32_t)nb, &bp->sub_bound, &bp->recb);
    bp->tseq = nullptr;
}

// Reserves the buffers bucket_prepare uses for this shape.
static int bucket_reserve(xtn_context* c, const BucketPlan& bp, int n, int d, uint64_t V) {
    if (bp.slotted) XTN_TRY(ensure(c->scur, sizeof(uint32_t) * bp.sub_bound));
    XTN_TRY(ensure(c->bcounts, sizeof(uint32_t) * (size_t)bp.ntiles * bp.nb));
    XTN_TRY(ensure(c->boffs, sizeof(uint32_t) * (size_t)bp.ntiles * bp.nb));
    XTN_TRY(ensure(c->btotals, sizeof(uint32_t) * (bp.nb + 1)));
    XTN_TRY(ensure(c->bstart, sizeof(uint64_t) * (bp.nb + 1)));
    if (bp.staged && d >= 2) {
        XTN_TRY(ensure(c->tcnt, sizeof(uint32_t) * n));
        XTN_TRY(ensure(c->toff, sizeof(uint64_t) * (n + 1)));
        // a sequence has at most kKeyLen runs, so at most kKeyLen tasks
        XTN_TRY(ensure(c->tseq, sizeof(uint32_t) * std::min<uint64_t>(V, (uint64_t)kKeyLen * n) + 16));
    }
    return XTN_SUCCESS;
}

// The generation tasks of the n sequences at d = 2 (counts, offsets toff, task -> sequence map);
// the buffers come from bucket_reserve.
static int build_task_map(xtn_context* c, int n, BucketPlan* bp) {
    cudaStream_t s = c->stream;
    XTN_LAUNCH("task_counts", k_task_counts<<<blocks_for(n), kThreads, 0, s>>>(P<uint64_t>(c->runinfo), n,
                                                                               P<uint32_t>(c->tcnt)));
    XTN_TRY(scan_u32_to_u64(c, P<uint32_t>(c->tcnt), P<uint64_t>(c->toff), n));
    XTN_LAUNCH("task_seq", k_task_seq<<<blocks_for(n, kTaskSeqThreads), kTaskSeqThreads, 0, s>>>(
                               P<uint64_t>(c->toff), n, P<uint32_t>(c->tseq)));
    bp->tseq = P<uint32_t>(c->tseq);
    return XTN_SUCCESS;
}

// one_round: the search keeps every record at once (no rounds, no shards), which the
// generate-then-partition first level (option flat_gen) needs: it holds all V records twice.
// abort (graph form, may be null): the generation does nothing when it is set.
static int bucket_prepare(xtn_context* c, int n, int d, uint64_t V, BucketPlan* bp, bool one_round = false,
                          const unsigned int* abort = nullptr) {
    cudaStream_t s = c->stream;
    bucket_shape(c, n, d, V, bp, one_round);
    const int b1 = bp->b1, nb = bp->nb, ntiles = bp->ntiles, tile = bp->tile;
    const bool tables = d <= 2 && c->key_tables;
    const size_t hist_smem = sizeof(uint32_t) * nb;
    XTN_TRY(bucket_reserve(c, *bp, n, d, V));
    XTN_TRY(bucket_attrs(c));
    if (bp->staged && d >= 2) XTN_TRY(build_task_map(c, n, bp));
    if (bp->flat) {
        // every record in sequence order into recB, with the per-tile histograms
        XTN_TRY(ensure(c->recA, sizeof(uint64_t) * V + 64));
        XTN_TRY(ensure(c->recB, sizeof(uint64_t) * bp->recb + 64));
        XTN_LAUNCH("bucket_gen", (k_bucket_gen<kBucketThreads, 2><<<ntiles, kBucketThreads, hist_smem, s>>>(
                                     P<uint8_t>(c->klen), P<uint64_t>(c->runinfo), P<uint64_t>(c->ktab),
                                     P<uint64_t>(c->voff), P<uint64_t>(c->toff), bp->tseq, n, tile, d, b1,
                                     id_bits_for(n), P<uint64_t>(c->recB), P<uint32_t>(c->bcounts), abort, 0, 0ull)));
    } else {
        XTN_LAUNCH("bucket_count", k_bucket_count<<<ntiles, kBucketThreads, hist_smem, s>>>(
                                       P<u128>(c->keys), P<uint8_t>(c->klen), P<uint64_t>(c->runinfo),
                                       tables ? P<uint64_t>(c->ktab) : nullptr, n, tile, d, b1, P<uint32_t>(c->bcounts)));
    }
    XTN_LAUNCH("bucket_colscan", k_bucket_colscan<<<(nb + 31) / 32, kColscanWarps * 32, 0, s>>>(
                                     P<uint32_t>(c->bcounts), ntiles, nb, P<uint32_t>(c->boffs), P<uint32_t>(c->btotals)));
    XTN_TRY(scan_u32_to_u64(c, P<uint32_t>(c->btotals), P<uint64_t>(c->bstart), nb));
    XTN_CK(cudaGetLastError());
    return XTN_SUCCESS;
}

// The split of the plan's jobs (recA -> recB): one CTA per bucket, or a cluster of
// split_slices CTAs per bucket, launched for every one of the b_n buckets without waiting for
// the plan: those past the plan's job count exit at once. The slotted split (bp.slotted) takes
// kSplitSlices independent CTAs per job and lists its sub-buckets afterwards.
// recs: the records of the b_n first-level buckets (a capacity in the graph form). The one-pass
// split takes the 8192-record stage when the buckets average 2^20 records or more (split_chunk 0)
// or when split_chunk is 8192: at 10M sequences (2.1M-record buckets) it took 5.27 against 5.44
// ms, at 1M (214k-record buckets, slices of 27k records) 0.57 against 0.49 ms.
static void launch_split(xtn_context* c, const BucketPlan& bp, uint32_t b_n, uint64_t sub_bound, size_t desc_cap,
                         uint64_t recs, const unsigned int* abort, cudaStream_t s) {
    if (bp.slotted) {
        cudaMemsetAsync(c->scur.p, 0, sizeof(uint32_t) * sub_bound, s);
        const bool huge = c->split_chunk == 8192 || (c->split_chunk == 0 && b_n > 0 && recs / b_n >= (uint64_t(1) << 20));
        if (huge)
            XTN_LAUNCH("bucket_split",
                       (k_bucket_split_slotted<StageHuge, kSplitSlices><<<b_n * kSplitSlices, StageHuge::kThreads,
                                                                         sizeof(StageSmem<StageHuge>), s>>>(
                           P<SplitJob>(c->bjobs), P<uint64_t>(c->recA), P<uint64_t>(c->recB), c->group_cap,
                           P<unsigned int>(c->scur), P<unsigned int>(c->bcnt), abort)));
        else
            XTN_LAUNCH("bucket_split",
                       (k_bucket_split_slotted<StageLarge, kSplitSlices><<<b_n * kSplitSlices, StageLarge::kThreads,
                                                                          sizeof(StageSmem<StageLarge>), s>>>(
                           P<SplitJob>(c->bjobs), P<uint64_t>(c->recA), P<uint64_t>(c->recB), c->group_cap,
                           P<unsigned int>(c->scur), P<unsigned int>(c->bcnt), abort)));
        XTN_LAUNCH("split_descs", k_split_slot_descs<<<b_n, 256, 0, s>>>(
                                      P<SplitJob>(c->bjobs), P<unsigned int>(c->scur), c->group_cap,
                                      P<BucketDesc>(c->bdesc), P<BucketDesc>(c->bfall), (uint32_t)desc_cap,
                                      P<unsigned int>(c->bcnt), abort));
        return;
    }
    const int sl = c->split_slices;
    const unsigned grid = b_n * (unsigned)sl;
#define XTN_SPLIT(CFG, SL)                                                                                         \
    XTN_LAUNCH("bucket_split", k_bucket_split_staged<CFG, SL><<<grid, CFG::kThreads, sizeof(StageSmem<CFG>), s>>>( \
                                   P<SplitJob>(c->bjobs), P<uint64_t>(c->recA), P<uint64_t>(c->recB), c->group_cap, \
                                   P<BucketDesc>(c->bdesc), P<BucketDesc>(c->bfall), (uint32_t)desc_cap,        \
                                   P<unsigned int>(c->bcnt)))
    if (c->split_chunk == 2048) {
        if (sl == kSplitSlices) XTN_SPLIT(SplitSmall, kSplitSlices);
        else XTN_SPLIT(SplitSmall, 1);
    } else {
        if (sl == kSplitSlices) XTN_SPLIT(StageLarge, kSplitSlices);
        else XTN_SPLIT(StageLarge, 1);
    }
#undef XTN_SPLIT
}

// The first-level partition of the records k_bucket_gen wrote in sequence order (recB -> recA).
static void launch_partition(xtn_context* c, const BucketPlan& bp, int n, int idbits, const unsigned int* abort,
                             cudaStream_t s) {
    XTN_LAUNCH("bucket_partition",
               k_bucket_partition<StageHuge><<<bp.ntiles, StageHuge::kThreads, sizeof(StageSmem<StageHuge>), s>>>(
                   P<uint64_t>(c->recB), P<uint64_t>(c->voff), n, bp.tile, bp.b1, idbits, P<uint32_t>(c->boffs),
                   P<uint64_t>(c->bstart), P<uint64_t>(c->recA), P<unsigned int>(c->bcnt), abort, 0, 0ull));
}

// The staged first-level scatter in the context's stage shape (stage_chunk 2048, 4096 or 8192).
static void launch_scatter_staged(xtn_context* c, const BucketPlan& bp, int n, int d, int idbits, uint32_t b_lo,
                                  uint32_t b_n, uint64_t base, const unsigned int* abort, cudaStream_t s) {
#define XTN_SCATTER(CFG)                                                                                          \
    XTN_LAUNCH("bucket_scatter",                                                                                 \
               k_bucket_scatter_staged<CFG><<<bp.ntiles, CFG::kThreads, sizeof(ScatterSmem<CFG>), s>>>(           \
                   P<uint8_t>(c->klen), P<uint64_t>(c->runinfo), P<uint64_t>(c->ktab), P<uint64_t>(c->voff),    \
                   P<uint64_t>(c->toff), bp.tseq, n, bp.tile, d, bp.b1, idbits, P<uint32_t>(c->boffs),         \
                   P<uint64_t>(c->bstart), b_lo, b_n, base, P<uint64_t>(c->recA), abort))
    if (bp.small) XTN_SCATTER(StageSmall);
    else if (c->stage_chunk == 8192) XTN_SCATTER(StageHuge);
    else XTN_SCATTER(StageLarge);
#undef XTN_SCATTER
}

// One round: the records of first-level buckets [b_lo, b_lo + b_n), which hold Vr records at
// global positions [base, base + Vr), are written to recA (positions minus base), oversized
// buckets split into recB, and every bucket grouped; the candidate pairs are written to `out`
// from index `at` (grown, keeping entries [0, at), when they do not fit). *Pc receives the
// number of candidates of the round.
static int bucket_round(xtn_context* c, const BucketPlan& bp, int n, int d, int idbits, uint32_t b_lo, uint32_t b_n,
                        uint64_t base, uint64_t Vr, DevBuf& out, uint64_t at, uint64_t* Pc,
                        bool first_level_done = false) {
    cudaStream_t s = c->stream;
    const int b1 = bp.b1, nb = bp.nb;
    uint64_t sub_bound = 0, recb = 0;
    slot_sizes(c, bp, Vr, b_n, &sub_bound, &recb);
    XTN_TRY(ensure(c->recA, sizeof(uint64_t) * Vr + 64));
    XTN_TRY(ensure(c->recB, sizeof(uint64_t) * recb + 64));
    if (bp.slotted) XTN_TRY(ensure(c->scur, sizeof(uint32_t) * sub_bound));
    const uint64_t* bstart = P<uint64_t>(c->bstart);
    XTN_TRY(ensure(c->bcnt, 64));
    XTN_CK(cudaMemsetAsync(c->bcnt.p, 0, 64, s));
    if (first_level_done) {
        // (recA and bstart hold the round's first-level buckets already: the shard exchange)
    } else if (bp.flat) {
        launch_partition(c, bp, n, idbits, nullptr, s);
    } else if (bp.staged) {
        launch_scatter_staged(c, bp, n, d, idbits, b_lo, b_n, base, nullptr, s);
    } else {
        XTN_LAUNCH("bucket_scatter", k_bucket_scatter<<<bp.ntiles, kBucketThreads, sizeof(uint32_t) * nb, s>>>(
                                         P<u128>(c->keys), P<uint8_t>(c->klen), n, bp.tile, d, b1, idbits,
                                         P<uint32_t>(c->boffs), bstart, b_lo, b_n, base, P<uint64_t>(c->recA),
                                         nullptr));
    }
    XTN_CK(cudaGetLastError());
    XTN_CK(cudaEventRecord(c->ev[2], s));

    // plan: buckets that fit go to grouping, the rest are split by ranges of the next hash bits
    const size_t desc_cap = (size_t)b_n * 3 + 4 * Vr / c->group_cap + 2048;
    XTN_TRY(ensure(c->bdesc, sizeof(BucketDesc) * desc_cap));
    XTN_TRY(ensure(c->bfall, sizeof(BucketDesc) * desc_cap));
    XTN_TRY(ensure(c->bjobs, sizeof(SplitJob) * b_n));
    XTN_LAUNCH("bucket_plan", k_bucket_plan<<<blocks_for(b_n), kThreads, 0, s>>>(
                                  bstart + b_lo, (int)b_n, base, c->group_cap, (uint32_t)c->split_fill, P<BucketDesc>(c->bdesc),
                                  (uint32_t)desc_cap, P<SplitJob>(c->bjobs), P<unsigned int>(c->bcnt), nullptr));
    XTN_CK(cudaGetLastError());
    uint32_t cnt[8] = {0};
    {
        launch_split(c, bp, b_n, sub_bound, desc_cap, Vr, nullptr, s);
        XTN_CK(cudaGetLastError());
        XTN_CK(cudaMemcpyAsync(c->h_scalar, c->bcnt.p, 32, cudaMemcpyDeviceToHost, s));
        XTN_CK(cudaStreamSynchronize(s));
        memcpy(cnt, c->h_scalar, 32);
        if (cnt[kCntWaitFail] != 0) {
            set_err("bucket partition or split: " + std::to_string(cnt[kCntWaitFail]) +
                    " chunk copies did not complete in time");
            return XTN_ERR_CUDA;
        }
        if (cnt[kCntDropped] != 0) {
            set_err("bucket plan: " + std::to_string(cnt[kCntDropped]) + " descriptors beyond the list capacity");
            return XTN_ERR_CUDA;
        }
    }
    XTN_CK(cudaEventRecord(c->ev[3], s));
    const uint32_t ndesc = cnt[kCntDesc];

    // group every listed bucket in shared memory; buckets with too many runs are appended
    // to the fallback list (counter kCntFallback); the cursor starts at `at`
    const uint64_t want =
        std::max<uint64_t>({c->last_pc_per_rec > 0 ? (uint64_t)(c->last_pc_per_rec * 1.25 * (double)Vr) : 0,
                            Vr / 16, (uint64_t)1 << 20});
    uint64_t cap = std::max<uint64_t>(at + want, out.cap / sizeof(uint64_t) > 8 ? out.cap / sizeof(uint64_t) - 8 : 0);
    uint64_t total = at;
    const uint32_t nfall_split = cnt[kCntFallback];
    for (int attempt = 0; attempt < 2; attempt++) {
        XTN_TRY(ensure_keep(c, out, sizeof(uint64_t) * cap + 64, sizeof(uint64_t) * at));
        XTN_LAUNCH("set_cursor", k_set_u64<<<1, 1, 0, s>>>(P<unsigned long long>(c->counter), (unsigned long long)at));
        XTN_CK(cudaMemsetAsync(P<unsigned long long>(c->counter) + 1, 0, 8, s));
        if (attempt > 0)  // the overflow list restarts after the split's fallback buckets
            XTN_LAUNCH("set_cursor", k_set_u64<<<1, 1, 0, s>>>(P<unsigned long long>(c->bcnt) + kCntFallback / 2,
                                                               ((unsigned long long)nfall_split << 32) | cnt[2]));
        if (ndesc > 0)
            XTN_TRY(launch_group(c, ndesc, c->group_persistent != 0 && ndesc > (uint32_t)c->sms * 8, idbits,
                                 P<uint64_t>(out), cap, (uint32_t)desc_cap, s));
        XTN_CK(cudaGetLastError());
        XTN_CK(cudaMemcpyAsync(c->h_scalar, c->counter.p, 16, cudaMemcpyDeviceToHost, s));
        XTN_CK(cudaMemcpyAsync(c->h_scalar + 2, c->bcnt.p, 32, cudaMemcpyDeviceToHost, s));
        XTN_CK(cudaStreamSynchronize(s));
        total = c->h_scalar[0];
        if ((c->h_scalar[1] & 0xffffffffu) != 0) {
            set_err("bucket grouping: a shared-memory bulk copy did not complete in time");
            return XTN_ERR_CUDA;
        }
        if ((uint32_t)c->h_scalar[5] != 0) {  // bcnt[kCntDropped]: low half of the fourth word
            set_err("bucket grouping: overflow list capacity exceeded");
            return XTN_ERR_CUDA;
        }
        if (total <= cap) break;
        cap = total;
    }
    const uint32_t nfall = (uint32_t)(c->h_scalar[3] >> 32);  // bcnt[kCntFallback]: high half of the second word
    c->stats.n_groups += ndesc;
    XTN_CK(cudaEventRecord(c->ev[4], s));

    // buckets too large for shared memory: gathered in batches (one kernel per batch), sorted
    // and grouped in global memory. Equal hashes lie in one bucket, so a batch of several
    // buckets groups exactly as the buckets one by one would (records of different first-level
    // buckets whose remaining hash fields agree add candidates that verification removes).
    if (nfall > 0) {
        std::vector<BucketDesc> fl(nfall);
        XTN_CK(cudaMemcpy(fl.data(), c->bfall.p, sizeof(BucketDesc) * nfall, cudaMemcpyDeviceToHost));
        uint64_t largest = 0;
        for (const BucketDesc& f : fl) largest = std::max<uint64_t>(largest, f.size);
        const uint64_t batch_cap = std::max<uint64_t>(largest, kFallbackBatchRecords);
        XTN_TRY(ensure(c->fbA, sizeof(uint64_t) * batch_cap + 64));
        XTN_TRY(ensure(c->fbB, sizeof(uint64_t) * batch_cap + 64));
        std::vector<uint64_t> offs;
        for (size_t b0 = 0; b0 < fl.size();) {
            size_t b1 = b0;
            uint64_t recs = 0;
            offs.clear();
            while (b1 < fl.size() && (b1 == b0 || recs + fl[b1].size <= batch_cap)) {
                offs.push_back(recs);
                recs += fl[b1].size;
                b1++;
            }
            offs.push_back(recs);
            XTN_TRY(ensure(c->scratch64, sizeof(uint64_t) * offs.size()));
            XTN_CK(cudaMemcpyAsync(c->scratch64.p, offs.data(), sizeof(uint64_t) * offs.size(), cudaMemcpyHostToDevice, s));
            XTN_LAUNCH("fallback_gather", k_fallback_gather<<<(unsigned)(b1 - b0), kThreads, 0, s>>>(
                                              P<BucketDesc>(c->bfall) + b0, P<uint64_t>(c->scratch64),
                                              P<uint64_t>(c->recA), P<uint64_t>(c->recB), P<uint64_t>(c->fbA)));
            uint64_t* sorted = nullptr;
            XTN_TRY(sort_u64(c, c->fbA, c->fbB, (int64_t)recs, idbits, 64, &sorted, XTN_SORT_NAMES("fallback_sort")));
            uint64_t more = 0;
            XTN_TRY(group_sorted(c, sorted, (int64_t)recs, idbits, out, total, &more));
            total += more;
            XTN_CK(cudaStreamSynchronize(s));  // offs (host) is refilled for the next batch
            b0 = b1;
        }
    }
    c->stats.n_fallback += nfall;
    *Pc = total - at;
    return XTN_SUCCESS;
}

// Single-round bucket engine: every record of the search in one pass.
static int candidates_bucketed(xtn_context* c, const BucketPlan& bp, int n, int d, int idbits, uint64_t V,
                               uint64_t* Pc) {
    return bucket_round(c, bp, n, d, idbits, 0, (uint32_t)bp.nb, 0, V, c->pairA, 0, Pc);
}

// Distinct non-self candidate pairs of pairA[0..Pc) into pairB[0..*U), in no particular order.
// Table size: dedup_first_slots (xtn_common.cuh). If an insertion runs past kDedupMaxProbes
// slots, the pass is repeated with dedup_regrow_slots under a new epoch.
static int dedup_pairs(xtn_context* c, uint64_t Pc, int idbits, uint64_t* U) {
    cudaStream_t s = c->stream;
    uint64_t want = c->dedup_slots_log2 ? (uint64_t(1) << c->dedup_slots_log2)
                                         : dedup_first_slots(Pc, c->dd_share, c->pair_dedup == 2);
    for (int attempt = 0; attempt < 3; attempt++) {
        const uint64_t T = pow2_at_least(want);
        if (c->dd_table.cap < sizeof(uint64_t) * T) {
            XTN_TRY(ensure(c->dd_table, sizeof(uint64_t) * T));
            XTN_CK(cudaMemsetAsync(c->dd_table.p, 0, c->dd_table.cap, s));
            c->dd_epoch = 0;
        }
        if (++c->dd_epoch >= (1u << kDedupTagBits)) {
            XTN_CK(cudaMemsetAsync(c->dd_table.p, 0, c->dd_table.cap, s));
            c->dd_epoch = 1;
        }
        XTN_CK(cudaMemsetAsync(c->counter.p, 0, 16, s));
        launch_pair_dedup(P<uint64_t>(c->pairA), (int64_t)Pc, idbits, P<unsigned long long>(c->dd_table), T,
                          (uint64_t)c->dd_epoch << kDedupKeyBits, P<uint64_t>(c->pairB), P<unsigned long long>(c->counter),
                          P<unsigned long long>(c->counter) + 1, nullptr, blocks_for((int64_t)Pc), s);
        XTN_CK(cudaGetLastError());
        XTN_CK(cudaMemcpyAsync(c->h_scalar, c->counter.p, 16, cudaMemcpyDeviceToHost, s));
        XTN_CK(cudaStreamSynchronize(s));
        if (c->h_scalar[1] == 0) {
            *U = c->h_scalar[0];
            c->dd_share = Pc ? std::max(0.01, (double)*U / (double)Pc) : 1.0;
            return XTN_SUCCESS;
        }
        want = dedup_regrow_slots(T, Pc);  // too full
    }
    set_err("candidate pair hash set: insertions did not find a free slot");
    return XTN_ERR_CUDA;
}

// ------------------------------------------------------------------ rounds
// A search whose variant records do not fit the memory budget (or a 32-bit position) runs in
// rounds, each over a contiguous range of first-level buckets. Equal variants hash to the same
// bucket, so every group of equal variants lies in one round; a candidate pair can still come
// from several rounds (through different shared variants), so the rounds' candidates go through
// one candidate-pair hash set that lives across the rounds: each distinct pair is appended to
// the distinct list once, by whichever round meets it first. This replaces the reference's
// lower-bound rounds over the min-id space (S/src/xtn.cu:383-470, cal_lowerbounds
// S/src/xtn.cu:179-184,218-230), which bound the candidate pairs held in host RAM; here the
// bound is on device memory, and the records are what grows with the input.
constexpr int kMaxShards = 1024;

struct Round {
    uint32_t b_lo, b_n;  // first-level buckets [b_lo, b_lo + b_n)
    uint64_t base, size; // their records: global positions [base, base + size)
};

// Device memory this context holds in its buffers.
static size_t held_bytes(const xtn_context* c) {
    const DevBuf* bufs[] = {&c->chars, &c->offs, &c->keys, &c->klen, &c->vcnt, &c->voff, &c->recA, &c->recB,
                            &c->gstart, &c->gsize, &c->gcnt, &c->goff, &c->pairA, &c->pairB, &c->pairA2, &c->dist,
                            &c->flag, &c->fpos, &c->scratch64, &c->scratch32, &c->out_pairs, &c->out_dist,
                            &c->out_freq, &c->bcounts, &c->boffs, &c->bdesc, &c->bfall, &c->fbA, &c->fbB,
                            &c->runinfo, &c->tcnt, &c->toff, &c->ktab, &c->tseq, &c->dd_table, &c->os_status};
    size_t t = 0;
    for (const DevBuf* b : bufs) t += b->cap;
    return t;
}

// The memory model: the largest number of variant records one round may hold. The reference
// sizes each of its stages from the free device memory with a 20% margin (S/src/xtn.cu:21-26,
// 64-157); here the budget is the context option memory_budget, or else 80% of the free device
// memory plus what the context already holds (free memory is queried only when one round of
// the search would need more than half of the device). Per record of a round: 16 bytes of
// record buffers and about 20 bytes per expected candidate (two candidate buffers with
// headroom); per search: the per-sequence arrays and about 48 bytes per expected distinct pair
// (distinct list, hash-set slots, sort buffer, verification and output). The expectations are
// the previous search's ratios (6% candidates per record and all of them distinct at first).
static uint64_t round_record_limit(xtn_context* c, int n, int d, uint64_t V) {
    const double cpr = c->last_pc_per_rec > 0 ? c->last_pc_per_rec : 0.06;
    const double share = std::min(1.0, 1.25 * c->dd_share);
    // (the slotted split's buffer B holds about 1 / split_fill of the records plus a slot per
    // first-level bucket: up to 1.75x the records)
    const double per_rec = (c->split_slotted ? 22.0 : 16.0) + 20.0 * cpr;
    const double fixed = (d <= 2 && c->key_tables ? 273.0 : 41.0) * (double)n;
    const double pairs = 48.0 * share * cpr * (double)V;
    double budget = (double)c->memory_budget;
    if (budget <= 0 && fixed + pairs + per_rec * (double)V > 0.5 * (double)c->total_mem) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) budget = 0.8 * (double)(free_b + held_bytes(c));
        else cudaGetLastError();
    }
    uint64_t lim = UINT64_MAX;
    if (budget > 0) {
        const double room = budget - fixed - pairs;
        lim = room > per_rec ? (uint64_t)(room / per_rec) : 1;
    }
    if (c->max_round_records > 0) lim = std::min<uint64_t>(lim, (uint64_t)c->max_round_records);
    return std::min<uint64_t>(lim, (uint64_t)UINT32_MAX - (uint64_t(1) << 20));  // 32-bit positions in a round
}

// Contiguous bucket ranges of at most `limit` records each (bucket starts read from the device).
// Sharding (options shard_count, shard_index): shard k of K covers the first-level buckets whose
// first record lies in [k V / K, (k + 1) V / K), so the shards hold about equal numbers of
// records and every group of equal hashes lies in exactly one shard.
static void shard_buckets(const std::vector<uint64_t>& bs, int nb, int k, int K, uint32_t* lo, uint32_t* hi) {
    const uint64_t V = bs[nb];
    auto bound = [&](int j) -> uint32_t {
        if (j >= K) return (uint32_t)nb;
        const uint64_t at = (uint64_t)((unsigned __int128)V * (unsigned)j / (unsigned)K);
        return (uint32_t)(std::lower_bound(bs.begin(), bs.begin() + nb, at) - bs.begin());
    };
    *lo = bound(k);
    *hi = std::max(*lo, bound(k + 1));
}

static int plan_rounds(xtn_context* c, const BucketPlan& bp, uint64_t limit, std::vector<Round>* rounds) {
    std::vector<uint64_t> bs(bp.nb + 1);
    XTN_CK(cudaMemcpyAsync(bs.data(), c->bstart.p, sizeof(uint64_t) * (bp.nb + 1), cudaMemcpyDeviceToHost, c->stream));
    XTN_CK(cudaStreamSynchronize(c->stream));
    rounds->clear();
    uint32_t lo = 0, end = (uint32_t)bp.nb;
    if (c->shard_count > 1) shard_buckets(bs, bp.nb, c->shard_index, c->shard_count, &lo, &end);
    while (lo < end) {
        if (bs[lo + 1] - bs[lo] > limit) {
            set_err("the memory budget cannot hold one first-level bucket (" + std::to_string(bs[lo + 1] - bs[lo]) +
                    " variant records, at most " + std::to_string(limit) + " per round)");
            return XTN_ERR_NOMEM;
        }
        uint32_t hi = lo + 1;
        while (hi < end && bs[hi + 1] - bs[lo] <= limit) hi++;
        rounds->push_back(Round{lo, hi - lo, bs[lo], bs[hi] - bs[lo]});
        lo = hi;
    }
    return XTN_SUCCESS;
}

// Candidate-pair hash set of a search: T slots (a power of two) of c->dd_table under a fresh
// epoch, cleared on `st` when the table is (re)allocated or the epoch wraps.
static int dedup_table(xtn_context* c, uint64_t want, cudaStream_t st, uint64_t* T, uint64_t* tag) {
    *T = pow2_at_least(want);
    if (c->dd_table.cap < sizeof(uint64_t) * *T) {
        XTN_TRY(ensure(c->dd_table, sizeof(uint64_t) * *T));
        XTN_CK(cudaMemsetAsync(c->dd_table.p, 0, c->dd_table.cap, st));
        c->dd_epoch = 0;
    }
    if (++c->dd_epoch >= (1u << kDedupTagBits)) {
        XTN_CK(cudaMemsetAsync(c->dd_table.p, 0, c->dd_table.cap, st));
        c->dd_epoch = 1;
    }
    *tag = (uint64_t)c->dd_epoch << kDedupKeyBits;
    return XTN_SUCCESS;
}

// Multi-round candidates. With the hash set, the distinct pairs of all rounds end in
// c->pairB[0..*U) (*distinct = true): round r's candidates are written to one of two buffers
// (pairA, pairA2) and de-duplicated on stream2 while round r + 1 generates and groups on the
// main stream (round_overlap; otherwise everything runs on the main stream in turn). Without
// the hash set (n > 2^24 or pair_dedup = 0) every round's candidates are appended to c->pairA
// (*U = *Ptotal, *distinct = false), to be sorted and checked for repeats afterwards.
static int candidates_rounds(xtn_context* c, const BucketPlan& bp, int n, int d, int idbits, uint64_t V,
                             const std::vector<Round>& rounds, uint64_t* Ptotal, uint64_t* U_out, bool* distinct) {
    cudaStream_t s = c->stream;
    uint64_t Ptot = 0;
    *distinct = c->pair_dedup && 2 * idbits <= kDedupKeyBits;
    if (rounds.empty()) {  // a shard without buckets
        *Ptotal = *U_out = 0;
        return XTN_SUCCESS;
    }
    if (!*distinct) {
        for (const Round& r : rounds) {
            uint64_t pc = 0;
            XTN_TRY(bucket_round(c, bp, n, d, idbits, r.b_lo, r.b_n, r.base, r.size, c->pairA, Ptot, &pc));
            Ptot += pc;
        }
        *Ptotal = *U_out = Ptot;
        return XTN_SUCCESS;
    }
    const bool overlap = c->round_overlap != 0;
    cudaStream_t sd = overlap ? c->stream2 : s;  // stream of the dedup passes
    DevBuf* cand[2] = {&c->pairA, overlap ? &c->pairA2 : &c->pairA};
    XTN_TRY(ensure(c->ddcnt, 64));
    XTN_CK(cudaMemsetAsync(c->ddcnt.p, 0, 64, s));  // distinct count, insertions that ran out of probes
    XTN_CK(cudaEventRecord(c->ev_round[0], s));
    XTN_CK(cudaStreamWaitEvent(sd, c->ev_round[0], 0));
    unsigned long long* n_uniq = P<unsigned long long>(c->ddcnt);
    uint64_t T = 0, tag = 0, Pc_est = 0, U_now = 0;
    uint64_t U_before[2] = {0, 0}, Pc_r[2] = {0, 0};
    auto launch_dedup = [&](int slot) -> int {
        if (Pc_r[slot] > 0)
            launch_pair_dedup(P<uint64_t>(*cand[slot]), (int64_t)Pc_r[slot], idbits, P<unsigned long long>(c->dd_table),
                              T, tag, P<uint64_t>(c->pairB), n_uniq, n_uniq + 1, nullptr,
                              blocks_for((int64_t)Pc_r[slot]), sd);
        XTN_CK(cudaGetLastError());
        XTN_CK(cudaMemcpyAsync(c->h_scalar + 8, c->ddcnt.p, 16, cudaMemcpyDeviceToHost, sd));
        return XTN_SUCCESS;
    };
    // waits for the dedup of the round in `slot`; when an insertion ran out of probes, the table
    // grows, is rebuilt from the distinct pairs of the earlier rounds, and the round is redone
    auto settle = [&](int slot) -> int {
        for (int attempt = 0;; attempt++) {
            XTN_CK(cudaStreamSynchronize(sd));
            if (c->h_scalar[9] == 0) {
                U_now = c->h_scalar[8];
                return XTN_SUCCESS;
            }
            if (attempt == 2) {
                set_err("candidate pair hash set: insertions did not find a free slot");
                return XTN_ERR_CUDA;
            }
            XTN_TRY(dedup_table(c, dedup_regrow_slots(T, Pc_est), sd, &T, &tag));
            XTN_LAUNCH("set_cursor", k_set_u64<<<1, 1, 0, sd>>>(n_uniq, (unsigned long long)U_before[slot]));
            XTN_CK(cudaMemsetAsync(n_uniq + 1, 0, 8, sd));
            if (U_before[slot] > 0)
                launch_pair_dedup(P<uint64_t>(c->pairB), (int64_t)U_before[slot], idbits,
                                  P<unsigned long long>(c->dd_table), T, tag, nullptr, n_uniq, n_uniq + 1, nullptr,
                                  blocks_for((int64_t)U_before[slot]), sd);
            XTN_TRY(launch_dedup(slot));
        }
    };
    for (size_t r = 0; r < rounds.size(); r++) {
        const int slot = (int)(r & 1);
        uint64_t pc = 0;
        XTN_TRY(bucket_round(c, bp, n, d, idbits, rounds[r].b_lo, rounds[r].b_n, rounds[r].base, rounds[r].size,
                             *cand[slot], 0, &pc));
        Ptot += pc;
        if (pc >= (uint64_t)UINT32_MAX) {
            set_err("too many candidate pairs in one round (" + std::to_string(pc) + ")");
            return XTN_ERR_LIMIT;
        }
        if (overlap && r > 0) XTN_TRY(settle(slot ^ 1));  // its buffer is the next round's
        if (r == 0) {
            // the table is sized for the whole search, extrapolated from the first round
            Pc_est = (uint64_t)((double)pc * (double)V / (double)std::max<uint64_t>(1, rounds[0].size) * 1.1) + 1;
            XTN_TRY(dedup_table(c, dedup_first_slots(Pc_est, c->dd_share, c->pair_dedup == 2), sd, &T, &tag));
        }
        // the distinct list grows by at most this round's candidates (the dedup stream is idle)
        XTN_TRY(ensure_keep(c, c->pairB, sizeof(uint64_t) * (U_now + pc) + 64, sizeof(uint64_t) * U_now));
        U_before[slot] = U_now;
        Pc_r[slot] = pc;
        XTN_CK(cudaEventRecord(c->ev_round[slot], s));
        XTN_CK(cudaStreamWaitEvent(sd, c->ev_round[slot], 0));
        XTN_TRY(launch_dedup(slot));
        if (!overlap) XTN_TRY(settle(slot));
    }
    if (overlap) XTN_TRY(settle((int)((rounds.size() - 1) & 1)));
    *Ptotal = Ptot;
    *U_out = U_now;
    c->dd_share = Ptot ? std::max(0.01, (double)U_now / (double)Ptot) : 1.0;
    return XTN_SUCCESS;
}

// The nearest-neighbour pipeline on device-resident input. rows (optional) maps search index
// -> CSR row. On success the result is in c->out_pairs / c->out_dist, c->n_out entries; the
// verified pair list in sorted (x, y) order of search indexes.
static int nn_tail(xtn_context* c, const uint8_t* chars, const uint32_t* offs, const int32_t* rows, int n, int d,
                   int measure, uint64_t Pc, bool distinct);
static int pack_and_count(xtn_context* c, const uint8_t* chars, const uint32_t* offs, const int32_t* rows, int n,
                          int d, bool validate, uint64_t* V_out);
static int nn_after_count(xtn_context* c, const uint8_t* chars, const uint32_t* offs, const int32_t* rows, int n,
                          int d, int measure, uint64_t V);

static int run_nn(xtn_context* c, const uint8_t* chars, const uint32_t* offs, const int32_t* rows, int n, int d,
                  int measure, bool validate) {
    xtn_stats& st = c->stats;
    memset(&st, 0, sizeof st);
    st.n_seqs = n;
    st.n_rounds = 1;
    const int idbits = id_bits_for(n);
    st.id_bits = idbits;
    cudaStream_t s = c->stream;
    XTN_CK(cudaEventRecord(c->ev[0], s));
    uint64_t V = 0;
    XTN_TRY(pack_and_count(c, chars, offs, rows, n, d, validate, &V));
    st.n_variants = (int64_t)V;
    if (c->shard_count > 1 && (c->engine != 0 || c->shard_index >= c->shard_count)) {
        set_err(c->engine != 0 ? "sharding needs the bucket engine (engine 0)"
                               : "shard_index must be below shard_count");
        return XTN_ERR_ARG;
    }
    if (c->engine == 1 && V >= (uint64_t)UINT32_MAX) {
        set_err("too many deletion variants for the sort engine's one round (" + std::to_string(V) + ")");
        return XTN_ERR_LIMIT;
    }
    return nn_after_count(c, chars, offs, rows, n, d, measure, V);
}

// Length check (validate), pack and variant offsets of a search; *V receives the variant count.
static int pack_and_count(xtn_context* c, const uint8_t* chars, const uint32_t* offs, const int32_t* rows, int n,
                          int d, bool validate, uint64_t* V_out) {
    cudaStream_t s = c->stream;
    if (validate) XTN_TRY(launch_length_check(c, offs, rows, n));

    // pack + variant counts
    XTN_TRY(ensure(c->keys, sizeof(u128) * n));
    XTN_TRY(ensure(c->klen, (size_t)n));
    XTN_TRY(ensure(c->vcnt, sizeof(uint32_t) * n));
    XTN_TRY(ensure(c->voff, sizeof(uint64_t) * (n + 1)));
    XTN_TRY(ensure(c->runinfo, sizeof(uint64_t) * n));
    const bool tables = d <= 2 && c->key_tables;
    if (tables) XTN_TRY(ensure(c->ktab, sizeof(uint64_t) * kTabLen * (size_t)n));
    XTN_LAUNCH("pack", k_pack<<<blocks_for(n, kPackThreads), kPackThreads, 0, s>>>(chars, offs, rows, n, d, P<u128>(c->keys), P<uint8_t>(c->klen),
                                             P<uint32_t>(c->vcnt), P<uint64_t>(c->runinfo),
                                             tables ? P<uint64_t>(c->ktab) : nullptr));
    XTN_CK(cudaGetLastError());
    XTN_TRY((scan_1p<uint32_t, uint64_t>(c, P<uint32_t>(c->vcnt), P<uint64_t>(c->voff), n, c->wait_fault_test)));
    c->wait_fault_test = 0;
    XTN_CK(cudaEventRecord(c->ev[1], s));
    uint64_t V = 0;
    if (validate) XTN_CK(cudaMemcpyAsync(c->h_scalar + 1, c->lencheck.p, 4, cudaMemcpyDeviceToHost, s));
    XTN_CK(cudaMemcpyAsync(c->h_scalar + 2, c->dev_err.p, 4, cudaMemcpyDeviceToHost, s));
    XTN_TRY(read_scalar(c, P<uint64_t>(c->voff) + n, 8, &V));
    if (validate) XTN_TRY(length_check_result(c, (uint32_t)c->h_scalar[1]));
    if ((uint32_t)c->h_scalar[2] != 0) {  // a look-back wait gave up: the offsets are unusable
        XTN_CK(cudaMemsetAsync(c->dev_err.p, 0, 16, s));
        XTN_CK(cudaStreamSynchronize(s));
        set_err(std::to_string((uint32_t)c->h_scalar[2]) +
                " look-back waits (radix sort or scan) did not complete in time");
        return XTN_ERR_CUDA;
    }
    *V_out = V;
    return XTN_SUCCESS;
}

// The search from its variant offsets on: candidate pairs (bucket or sort engine, in rounds
// when needed), then nn_tail.
static int nn_after_count(xtn_context* c, const uint8_t* chars, const uint32_t* offs, const int32_t* rows, int n,
                          int d, int measure, uint64_t V) {
    xtn_stats& st = c->stats;
    const int idbits = id_bits_for(n);

    // candidate pairs: every (min id, max id) of every group of equal variant hashes
    uint64_t Pc = 0;
    XTN_TRY(ensure(c->counter, 64));
    bool distinct = false;  // pairB already holds the distinct pairs (multi-round search)
    if (c->engine == 1) {
        XTN_TRY(candidates_sorted(c, n, d, idbits, V, &Pc));
    } else {
        BucketPlan bp;
        const uint64_t limit = round_record_limit(c, n, d, V);
        const bool one_round = V <= limit && c->shard_count <= 1;
        XTN_TRY(bucket_prepare(c, n, d, V, &bp, one_round));
        if (one_round) {
            XTN_TRY(candidates_bucketed(c, bp, n, d, idbits, V, &Pc));
        } else {
            std::vector<Round> rounds;
            XTN_TRY(plan_rounds(c, bp, limit, &rounds));
            st.n_rounds = (int32_t)rounds.size();
            uint64_t U = 0;
            XTN_TRY(candidates_rounds(c, bp, n, d, idbits, V, rounds, &Pc, &U, &distinct));
            if (distinct) {
                st.n_candidates = (int64_t)Pc;
                c->last_pc_per_rec = V ? (double)Pc / (double)V : 0.0;
                Pc = U;
            }
        }
    }
    if (!distinct) {
        c->last_pc_per_rec = V ? (double)Pc / (double)V : 0.0;
        st.n_candidates = (int64_t)Pc;
    }
    return nn_tail(c, chars, offs, rows, n, d, measure, Pc, distinct);
}

// The end of a nearest-neighbour search once its candidate pairs are known: Pc candidates in
// c->pairA (distinct = false), or Pc distinct pairs in c->pairB (distinct = true, rounds); the
// candidates are de-duplicated (hash set), sorted, verified and compacted into the context's
// result. The statistics' stage times run from event 0, recorded by the caller.
static int nn_tail(xtn_context* c, const uint8_t* chars, const uint32_t* offs, const int32_t* rows, int n, int d,
                   int measure, uint64_t Pc, bool distinct) {
    xtn_stats& st = c->stats;
    cudaStream_t s = c->stream;
    const int idbits = id_bits_for(n);
    if (Pc >= (uint64_t)UINT32_MAX) {
        set_err("too many " + std::string(distinct ? "distinct" : "candidate") + " pairs (" + std::to_string(Pc) + ")");
        return XTN_ERR_LIMIT;
    }
    if (distinct) {
        XTN_TRY(ensure(c->pairA, sizeof(uint64_t) * Pc + 64));  // the sort's second buffer
    } else {
        XTN_TRY(ensure_keep(c, c->pairA, sizeof(uint64_t) * Pc + 64, sizeof(uint64_t) * Pc));
        XTN_TRY(ensure(c->pairB, sizeof(uint64_t) * Pc + 64));
    }
    XTN_CK(cudaEventRecord(c->ev[5], s));
    uint64_t* pairs = P<uint64_t>(c->pairA);
    if (distinct) {
        // the rounds' distinct pairs (pairB): only sorted and verified
        st.n_unique = (int64_t)Pc;
        pairs = P<uint64_t>(c->pairB);
        if (Pc > 1)
            XTN_TRY(sort_u64(c, c->pairB, c->pairA, (int64_t)Pc, 0, 2 * idbits, &pairs, XTN_SORT_NAMES("pair_sort")));
    } else if (c->pair_dedup && (int64_t)Pc >= kDedupMinPairs && 2 * idbits <= kDedupKeyBits) {
        // from here on Pc counts the distinct pairs (in pairB), which alone are sorted and verified
        XTN_TRY(dedup_pairs(c, Pc, idbits, &Pc));
        st.n_unique = (int64_t)Pc;
        pairs = P<uint64_t>(c->pairB);
        if (Pc > 1)
            XTN_TRY(sort_u64(c, c->pairB, c->pairA, (int64_t)Pc, 0, 2 * idbits, &pairs, XTN_SORT_NAMES("pair_sort")));
    } else if (Pc > 1) {
        XTN_TRY(sort_u64(c, c->pairA, c->pairB, (int64_t)Pc, 0, 2 * idbits, &pairs, XTN_SORT_NAMES("pair_sort")));
    }
    XTN_CK(cudaEventRecord(c->ev[6], s));

    // verify + compact
    XTN_TRY(ensure(c->dist, (size_t)Pc));
    XTN_TRY(ensure(c->flag, (size_t)Pc));
    XTN_TRY(ensure(c->fpos, sizeof(uint32_t) * (Pc + 1)));
    uint64_t nout = 0;
    if (Pc > 0) {
        launch_verify(c->verify_per, pairs, (int64_t)Pc, idbits, chars, offs, rows, d, measure, P<int8_t>(c->dist),
                      P<uint8_t>(c->flag), nullptr, s);
        XTN_CK(cudaGetLastError());
        XTN_TRY((scan_1p<uint8_t, uint32_t>(c, P<uint8_t>(c->flag), P<uint32_t>(c->fpos), (int64_t)Pc)));
        XTN_CK(cudaEventRecord(c->ev[7], s));
        // the output arrays hold every candidate, so the verified count (fpos[Pc]) is only read
        // with the final synchronisation
        XTN_TRY(ensure(c->out_pairs, sizeof(xtn_int2) * Pc));
        XTN_TRY(ensure(c->out_dist, (size_t)Pc));
        XTN_LAUNCH("compact", k_compact<<<blocks_for((int64_t)Pc), kThreads, 0, s>>>(pairs, (int64_t)Pc, idbits, P<int8_t>(c->dist),
                                                               P<uint8_t>(c->flag), P<uint32_t>(c->fpos),
                                                               P<xtn_int2>(c->out_pairs), P<int8_t>(c->out_dist), nullptr));
        c->h_scalar[6] = 0;
        XTN_CK(cudaMemcpyAsync(c->h_scalar + 6, P<uint32_t>(c->fpos) + Pc, 4, cudaMemcpyDeviceToHost, s));
    } else {
        XTN_CK(cudaEventRecord(c->ev[7], s));
    }
    XTN_CK(cudaGetLastError());
    XTN_CK(cudaEventRecord(c->ev[8], s));
    if (c->dev_err.p) XTN_CK(cudaMemcpyAsync(c->h_scalar + 7, c->dev_err.p, 8, cudaMemcpyDeviceToHost, s));
    XTN_CK(cudaStreamSynchronize(s));
    if (Pc > 0) nout = c->h_scalar[6];
    if (c->dev_err.p && (uint32_t)c->h_scalar[7] != 0) {
        XTN_CK(cudaMemsetAsync(c->dev_err.p, 0, 16, s));
        set_err(std::to_string((uint32_t)c->h_scalar[7]) +
                " look-back waits (radix sort or scan) did not complete in time");
        return XTN_ERR_CUDA;
    }
    c->n_out = (int64_t)nout;
    c->overlap_result = false;
    st.n_out = (int64_t)nout;
    // unique candidates = number of distinct pairs; counted from the verify flags' input side
    float ms = 0;
    for (int k = 0; k < S_COUNT; k++) {
        // a stage that a search form skips leaves its event unrecorded: its time reads as 0,
        // and the query's error is cleared so that no later cudaGetLastError reports it
        if (cudaEventElapsedTime(&ms, c->ev[k], c->ev[k + 1]) != cudaSuccess) {
            ms = 0;
            (void)cudaGetLastError();
        }
        st.ms_stage[k] = ms;
    }
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[S_COUNT]);
    st.ms_total = ms;
    return XTN_SUCCESS;
}

// ------------------------------------------------------------------ graph form
// The batched/persistent form of a search on device-resident inputs: the whole single-round
// launch sequence (length check, pack, variant offsets, count, scatter, plan, split, grouping
// by persistent CTAs that take bucket descriptors from a device-side queue, candidate-pair
// dedup, sort, verification, compaction) is captured once into a CUDA graph and replayed, with
// every data-dependent size read on the device. Buffers are sized from the previous plain
// search on the same input with headroom; the host reads one status block per replay. A replay
// that outgrows a capacity, meets a bucket too large for shared memory or a hash set too full,
// is redone by the plain form, which also re-sizes the graph. The plain form
// (run_nn) waits for the device four times per search to size its buffers and grids.
using GraphSig = std::array<int64_t, 13>;

struct GraphState {
    const uint8_t* chars = nullptr;
    const uint32_t* offs = nullptr;
    const int32_t* rows = nullptr;            // sequence i is row rows[i] (overlap: one row per unique string)
    const unsigned int* pre_abort = nullptr;  // an abort word set by stages captured before the search
    int n = 0, d = 0, measure = 0;
    GraphSig sig{};                  // options the capture depends on
    uint64_t Vcap = 0, Pcap = 0, Ucap = 0, T = 0;
    int b1 = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t* result = nullptr;      // where the sorted distinct pairs end (pairB or pairA)
    int64_t launches = 0;
    DevBuf status, table, os_status;
    uint32_t os_epoch = 0;
    std::vector<const void*> bufs;   // the context's buffers at capture (a reallocation invalidates it)
};

// Status block of one replay (device words, copied to the pinned host scalars 16..31).
enum {
    GS_V, GS_ABORT, GS_LENBAD, GS_CAND, GS_GROUP_ERR, GS_SPLIT_ERR, GS_DROPPED, GS_FALLBACK, GS_UNIQUE,
    GS_FULL, GS_LOOKBACK_ERR, GS_OUT, GS_NDESC, GS_WORDS
};

// Sets the abort word when the variant records exceed their capacity, a length is invalid or an
// earlier stage aborted.
__global__ void k_graph_guard(const uint64_t* __restrict__ V, uint64_t Vcap, const unsigned int* __restrict__ lenbad,
                              const unsigned int* __restrict__ pre, unsigned int* __restrict__ abort) {
    *abort = (*V > Vcap || *lenbad != 0xffffffffu || (pre && *pre)) ? 1u : 0u;
}

__global__ void k_graph_status(const uint64_t* __restrict__ V, const unsigned int* __restrict__ abort,
                               const unsigned int* __restrict__ lenbad, const unsigned long long* __restrict__ cursor,
                               const unsigned int* __restrict__ bcnt, const unsigned long long* __restrict__ ddcnt,
                               const unsigned int* __restrict__ dev_err, const uint32_t* __restrict__ fpos,
                               uint64_t Ucap, uint64_t* __restrict__ st) {
    const unsigned long long U = ddcnt[0];
    st[GS_V] = *V;
    st[GS_ABORT] = *abort;
    st[GS_LENBAD] = *lenbad;
    st[GS_CAND] = cursor[0];
    st[GS_GROUP_ERR] = reinterpret_cast<const unsigned int*>(cursor)[2];
    st[GS_SPLIT_ERR] = bcnt[kCntWaitFail];
    st[GS_DROPPED] = bcnt[kCntDropped];
    st[GS_FALLBACK] = bcnt[kCntFallback];
    st[GS_UNIQUE] = U;
    st[GS_FULL] = ddcnt[1];
    st[GS_LOOKBACK_ERR] = dev_err ? *dev_err : 0u;
    st[GS_OUT] = fpos[U < Ucap ? U : Ucap];
    st[GS_NDESC] = bcnt[kCntDesc];
}

// The options a capture depends on.
static GraphSig graph_signature(const xtn_context* c) {
    return GraphSig{c->stage_chunk,  c->split_chunk,  c->bucket_bits_max,     (int64_t)c->group_cap,
                    c->group_tma,    c->key_tables,   c->split_slices,        c->scatter_ctas_per_sm,
                    c->pair_dedup,   c->verify_per,   c->flat_gen,            c->split_fill,
                    c->split_slotted};
}

static void graph_release(GraphState* g) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    g->exec = nullptr;
    g->graph = nullptr;
}

// Enqueues the whole search for the capacities in g (no host waits, no allocations: every
// buffer is reserved beforehand).
static int graph_enqueue(xtn_context* c, GraphState* g) {
    cudaStream_t s = c->stream;
    const int n = g->n, d = g->d;
    const int idbits = id_bits_for(n);
    const bool tables = d <= 2 && c->key_tables;
    unsigned int* abort = P<unsigned int>(c->lencheck) + 1;
    XTN_CK(cudaMemsetAsync(c->lencheck.p, 0xff, 4, s));
    XTN_LAUNCH("check_lengths", k_check_lengths<<<blocks_for(n), kThreads, 0, s>>>(g->offs, g->rows, n,
                                                                                    P<unsigned int>(c->lencheck)));
    XTN_LAUNCH("pack", k_pack<<<blocks_for(n, kPackThreads), kPackThreads, 0, s>>>(
                           g->chars, g->offs, g->rows, n, d, P<u128>(c->keys), P<uint8_t>(c->klen), P<uint32_t>(c->vcnt),
                           P<uint64_t>(c->runinfo), tables ? P<uint64_t>(c->ktab) : nullptr));
    XTN_TRY((scan_1p<uint32_t, uint64_t>(c, P<uint32_t>(c->vcnt), P<uint64_t>(c->voff), n)));
    XTN_LAUNCH("graph_guard", k_graph_guard<<<1, 1, 0, s>>>(P<uint64_t>(c->voff) + n, g->Vcap,
                                                            P<unsigned int>(c->lencheck), g->pre_abort, abort));
    BucketPlan bp;
    XTN_TRY(bucket_prepare(c, n, d, g->Vcap, &bp, true, abort));
    if (bp.b1 != g->b1) {
        set_err("graph capture: first-level bucket bits changed");
        return XTN_ERR_CUDA;
    }
    const int nb = bp.nb;
    const uint64_t* bstart = P<uint64_t>(c->bstart);
    XTN_CK(cudaMemsetAsync(c->bcnt.p, 0, 64, s));
    if (bp.flat) {
        launch_partition(c, bp, n, idbits, abort, s);
    } else if (bp.staged) {
        launch_scatter_staged(c, bp, n, d, idbits, 0u, (uint32_t)nb, 0ull, abort, s);
    } else {
        XTN_LAUNCH("bucket_scatter", k_bucket_scatter<<<bp.ntiles, kBucketThreads, sizeof(uint32_t) * nb, s>>>(
                                         P<u128>(c->keys), P<uint8_t>(c->klen), n, bp.tile, d, bp.b1, idbits,
                                         P<uint32_t>(c->boffs), bstart, 0u, (uint32_t)nb, 0ull, P<uint64_t>(c->recA),
                                         abort));
    }
    const size_t desc_cap = (size_t)nb * 3 + 4 * g->Vcap / c->group_cap + 2048;
    XTN_LAUNCH("bucket_plan", k_bucket_plan<<<blocks_for(nb), kThreads, 0, s>>>(
                                  bstart, nb, 0ull, c->group_cap, (uint32_t)c->split_fill, P<BucketDesc>(c->bdesc), (uint32_t)desc_cap,
                                  P<SplitJob>(c->bjobs), P<unsigned int>(c->bcnt), abort));
    launch_split(c, bp, (uint32_t)nb, bp.sub_bound, desc_cap, g->Vcap, abort, s);
    XTN_LAUNCH("set_cursor", k_set_u64<<<1, 1, 0, s>>>(P<unsigned long long>(c->counter), 0ull));
    XTN_CK(cudaMemsetAsync(P<unsigned long long>(c->counter) + 1, 0, 8, s));
    XTN_TRY(launch_group(c, 0, true, idbits, P<uint64_t>(c->pairA), g->Pcap, (uint32_t)desc_cap, s));
    // candidate pairs -> distinct pairs (the table is cleared every replay: a fixed epoch)
    unsigned long long* ddcnt = P<unsigned long long>(c->ddcnt);
    XTN_CK(cudaMemsetAsync(c->ddcnt.p, 0, 16, s));
    XTN_CK(cudaMemsetAsync(g->table.p, 0, sizeof(uint64_t) * g->T, s));
    launch_pair_dedup(P<uint64_t>(c->pairA), (int64_t)g->Pcap, idbits, P<unsigned long long>(g->table), g->T,
                      1ull << kDedupKeyBits, P<uint64_t>(c->pairB), ddcnt, ddcnt + 1, P<unsigned long long>(c->counter),
                      (unsigned)std::min<int64_t>(blocks_for((int64_t)g->Pcap), (int64_t)c->sms * 16), s);
    uint64_t* pairs = P<uint64_t>(c->pairB);
    pairs = onesweep_sort_u64(P<uint64_t>(c->pairB), P<uint64_t>(c->pairA), (int64_t)g->Ucap, 0, 2 * idbits,
                              P<uint32_t>(c->os_scratch), P<unsigned long long>(g->os_status),
                              (int64_t)(g->os_status.cap / 8), &g->os_epoch, P<unsigned int>(c->dev_err), c->sms, s,
                              "pair_sort_hist", "pair_sort_pass", ddcnt);
    g->result = pairs;
    launch_verify(c->verify_per, pairs, (int64_t)g->Ucap, idbits, g->chars, g->offs, g->rows, d, g->measure,
                  P<int8_t>(c->dist), P<uint8_t>(c->flag), ddcnt, s);
    scan_exclusive_1p<uint8_t, uint32_t>(P<uint8_t>(c->flag), P<uint32_t>(c->fpos), (int64_t)g->Ucap,
                                         P<unsigned long long>(c->scan_status), P<unsigned int>(c->dev_err), s,
                                         c->wait_polls, 0, ddcnt);
    XTN_LAUNCH("compact", k_compact<<<blocks_for((int64_t)g->Ucap), kThreads, 0, s>>>(
                              pairs, (int64_t)g->Ucap, idbits, P<int8_t>(c->dist), P<uint8_t>(c->flag),
                              P<uint32_t>(c->fpos), P<xtn_int2>(c->out_pairs), P<int8_t>(c->out_dist), ddcnt));
    XTN_LAUNCH("graph_status", k_graph_status<<<1, 1, 0, s>>>(
                                   P<uint64_t>(c->voff) + n, abort, P<unsigned int>(c->lencheck),
                                   P<unsigned long long>(c->counter), P<unsigned int>(c->bcnt), ddcnt,
                                   P<unsigned int>(c->dev_err), P<uint32_t>(c->fpos), g->Ucap, P<uint64_t>(g->status)));
    XTN_CK(cudaMemcpyAsync(c->h_scalar + 16, g->status.p, sizeof(uint64_t) * GS_WORDS, cudaMemcpyDeviceToHost, s));
    XTN_CK(cudaGetLastError());
    return XTN_SUCCESS;
}

// Capacities from the plain search just run on this input (its statistics), every buffer the
// capture uses reserved. XTN_ERR_LIMIT: the input stays in the plain form.
static int graph_reserve(xtn_context* c, GraphState* g, const uint8_t* chars, const uint32_t* offs, const int32_t* rows,
                         int n, int d, int measure) {
    const xtn_stats& st = c->stats;
    if (c->engine != 0 || st.n_rounds != 1 || c->shard_count > 1 || !c->pair_dedup || 2 * id_bits_for(n) > kDedupKeyBits)
        return XTN_ERR_LIMIT;
    g->chars = chars;
    g->offs = offs;
    g->rows = rows;
    g->pre_abort = nullptr;
    g->n = n;
    g->d = d;
    g->measure = measure;
    g->sig = graph_signature(c);
    const uint64_t V = (uint64_t)st.n_variants, Pc = (uint64_t)st.n_candidates;
    const uint64_t U = st.n_unique > 0 ? (uint64_t)st.n_unique : Pc;
    g->Vcap = V + V / 32 + 4096;
    g->Pcap = Pc + Pc / 8 + 65536;
    g->Ucap = std::min<uint64_t>(g->Pcap, U + U / 4 + 65536);
    if (g->Ucap > (uint64_t)kOsMaxKeys || g->Vcap >= (uint64_t)UINT32_MAX || g->Pcap >= (uint64_t)UINT32_MAX)
        return XTN_ERR_LIMIT;
    g->T = pow2_at_least(2 * g->Ucap);
    // the first-level shape the capacity implies, and every buffer reserved (the capture must
    // not allocate)
    BucketPlan bp;
    bucket_shape(c, n, d, g->Vcap, &bp, true);
    g->b1 = bp.b1;
    XTN_TRY(bucket_reserve(c, bp, n, d, g->Vcap));
    const int nb = bp.nb;
    const size_t desc_cap = (size_t)nb * 3 + 4 * g->Vcap / c->group_cap + 2048;
    XTN_TRY(ensure(c->lencheck, 16));
    XTN_TRY(ensure(c->recA, sizeof(uint64_t) * g->Vcap + 64));
    XTN_TRY(ensure(c->recB, sizeof(uint64_t) * bp.recb + 64));
    XTN_TRY(ensure(c->bdesc, sizeof(BucketDesc) * desc_cap));
    XTN_TRY(ensure(c->bfall, sizeof(BucketDesc) * desc_cap));
    XTN_TRY(ensure(c->bjobs, sizeof(SplitJob) * nb));
    XTN_TRY(ensure(c->bcnt, 64));
    XTN_TRY(ensure(c->counter, 64));
    XTN_TRY(ensure(c->ddcnt, 64));
    XTN_TRY(ensure(c->pairA, sizeof(uint64_t) * g->Pcap + 64));
    XTN_TRY(ensure(c->pairB, sizeof(uint64_t) * g->Pcap + 64));
    XTN_TRY(ensure(c->dist, (size_t)g->Ucap + 64));
    XTN_TRY(ensure(c->flag, (size_t)g->Ucap + 64));
    XTN_TRY(ensure(c->fpos, sizeof(uint32_t) * (g->Ucap + 1)));
    // the plain search's result (c->n_out entries) is still to be read by the caller
    XTN_TRY(ensure_keep(c, c->out_pairs, sizeof(xtn_int2) * g->Ucap + 64, sizeof(xtn_int2) * (size_t)c->n_out));
    XTN_TRY(ensure_keep(c, c->out_dist, (size_t)g->Ucap + 64, (size_t)c->n_out));
    XTN_TRY(ensure(c->os_scratch, sizeof(uint32_t) * kOsScratchWords));
    XTN_TRY(ensure_err_word(c));
    XTN_TRY(ensure(c->scan_status, sizeof(unsigned long long) * scan_1p_words((int64_t)std::max<uint64_t>(g->Ucap, n))));
    XTN_TRY(ensure(g->status, sizeof(uint64_t) * GS_WORDS));
    XTN_TRY(ensure(g->table, sizeof(uint64_t) * g->T));
    XTN_TRY(ensure(g->os_status, sizeof(unsigned long long) * (size_t)onesweep_status_words((int64_t)g->Ucap)));
    XTN_TRY(bucket_attrs(c));
    return XTN_SUCCESS;
}

// Captures what enqueue() launches on the context's stream (launches counted, no per-launch
// events).
template <class F>
static int capture(xtn_context* c, F&& enqueue, cudaGraph_t* out, int64_t* launches) {
    XTN_CK(cudaStreamSynchronize(c->stream));
    KernelProfiler counting;
    KernelProfiler* saved = current_profiler();
    current_profiler() = &counting;
    XTN_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int r = enqueue();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    current_profiler() = saved;
    if (r != XTN_SUCCESS || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        if (r == XTN_SUCCESS) set_err(std::string("graph capture failed: ") + cudaGetErrorString(e));
        return r != XTN_SUCCESS ? r : XTN_ERR_CUDA;
    }
    *out = graph;
    *launches = counting.launches;
    return XTN_SUCCESS;
}

// Every device buffer of the context: a graph holds their addresses, so it is replayed only while
// none of them has been reallocated (by a search of another input, or by another form).
static std::vector<const void*> context_buffer_ptrs(const xtn_context* c);

// Capacities from the plain search just run on this input, buffers reserved, graph captured.
static int graph_build(xtn_context* c, GraphState* g, const uint8_t* chars, const uint32_t* offs, int n, int d,
                       int measure) {
    graph_release(g);
    XTN_TRY(graph_reserve(c, g, chars, offs, nullptr, n, d, measure));
    cudaGraph_t graph = nullptr;
    XTN_TRY(capture(c, [&] { return graph_enqueue(c, g); }, &graph, &g->launches));
    g->graph = graph;
    XTN_CK(cudaGraphInstantiate(&g->exec, graph, 0));
    g->bufs = context_buffer_ptrs(c);
    return XTN_SUCCESS;
}

// One replay of a captured form, timed with events; the statistics are reset (ms_total set).
static int graph_launch(xtn_context* c, cudaGraphExec_t exec) {
    cudaStream_t s = c->stream;
    xtn_stats& st = c->stats;
    memset(&st, 0, sizeof st);
    XTN_CK(cudaEventRecord(c->ev[0], s));
    XTN_CK(cudaGraphLaunch(exec, s));
    XTN_CK(cudaEventRecord(c->ev[8], s));
    XTN_CK(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[8]);
    st.ms_total = ms;
    return XTN_SUCCESS;
}

// The search's status block of a replay (host scalars 16..28) into the statistics and the result
// count; *redo is set when the plain form has to run instead.
static int graph_check(xtn_context* c, GraphState* g, bool* redo) {
    cudaStream_t s = c->stream;
    xtn_stats& st = c->stats;
    st.n_seqs = g->n;
    st.n_rounds = 1;
    st.id_bits = id_bits_for(g->n);
    const uint64_t* h = c->h_scalar + 16;
    *redo = false;
    if ((uint32_t)h[GS_LENBAD] != 0xffffffffu) return length_check_result(c, (uint32_t)h[GS_LENBAD]);
    if (h[GS_GROUP_ERR] || h[GS_SPLIT_ERR] || h[GS_LOOKBACK_ERR]) {
        XTN_CK(cudaMemsetAsync(c->dev_err.p, 0, 16, s));
        XTN_CK(cudaStreamSynchronize(s));
        set_err("graph form: a bounded device wait did not complete in time");
        return XTN_ERR_CUDA;
    }
    if (h[GS_DROPPED]) {
        set_err("graph form: descriptors beyond the list capacity");
        return XTN_ERR_CUDA;
    }
    if (h[GS_ABORT] || h[GS_CAND] > g->Pcap || h[GS_FALLBACK] || h[GS_FULL] || h[GS_UNIQUE] > g->Ucap) {
        *redo = true;  // a capacity or a shared-memory bound was exceeded
        return XTN_SUCCESS;
    }
    st.n_variants = (int64_t)h[GS_V];
    st.n_groups = (int64_t)h[GS_NDESC];
    st.n_candidates = (int64_t)h[GS_CAND];
    st.n_unique = (int64_t)h[GS_UNIQUE];
    st.n_out = (int64_t)h[GS_OUT];
    st.n_launches = g->launches;
    c->n_out = st.n_out;
    c->overlap_result = false;
    return XTN_SUCCESS;
}

// One search by the graph form; *redo is set when the plain form has to run instead.
static int graph_replay(xtn_context* c, GraphState* g, bool* redo) {
    XTN_TRY(graph_launch(c, g->exec));
    return graph_check(c, g, redo);
}

// The device-resident search in the graph form (option "graph" = 1).
static int nn_graph(xtn_context* c, const uint8_t* chars, const uint32_t* offs, int n, int d, int measure) {
    if (!c->graph) c->graph = new GraphState();
    GraphState* g = static_cast<GraphState*>(c->graph);
    const bool same = g->exec && g->chars == chars && g->offs == offs && g->n == n && g->d == d &&
                      g->measure == measure && g->sig == graph_signature(c) && g->bufs == context_buffer_ptrs(c);
    if (same) {
        bool redo = false;
        XTN_TRY(graph_replay(c, g, &redo));
        if (!redo) return XTN_SUCCESS;
    }
    // the plain form, then a graph sized from it for the next search on this input
    begin_run(c);
    int r = run_nn(c, chars, offs, nullptr, n, d, measure, true);
    end_run(c);
    if (r != XTN_SUCCESS) return r;
    const xtn_stats keep = c->stats;
    const int64_t keep_out = c->n_out;
    const int b = graph_build(c, g, chars, offs, n, d, measure);
    if (b != XTN_SUCCESS && b != XTN_ERR_LIMIT) return b;
    if (b == XTN_ERR_LIMIT) graph_release(g);  // this input stays in the plain form
    c->stats = keep;
    c->n_out = keep_out;
    return XTN_SUCCESS;
}

static int check_args(const xtn_args* a) {
    if (!a) {
        set_err("null args");
        return XTN_ERR_ARG;
    }
    if (a->distance < 1) {
        set_err("distance must be a valid number larger than 0");
        return XTN_ERR_ARG;
    }
    if (a->measure != XTN_LEVENSHTEIN && a->measure != XTN_HAMMING) {
        set_err("invalid measure option");
        return XTN_ERR_ARG;
    }
    return XTN_SUCCESS;
}

// Every sequence must have 1..kMaxInputLength residues (first_bad_offset: a threaded scan).
static int check_offsets(const uint32_t* offs, int n) {
    const int i = first_bad_offset(offs, n);
    if (i < 0) return XTN_SUCCESS;
    set_err("sequence " + std::to_string(i) + " has an invalid length");
    return XTN_ERR_ARG;
}

static int upload(xtn_context* c, const char* seqs, const uint32_t* offsets, int n) {
    size_t nch = offsets[n];
    XTN_TRY(ensure(c->chars, nch + 16));
    XTN_TRY(ensure(c->offs, sizeof(uint32_t) * (n + 1)));
    XTN_CK(cudaMemcpyAsync(c->chars.p, seqs, nch, cudaMemcpyHostToDevice, c->stream));
    XTN_CK(cudaMemcpyAsync(c->offs.p, offsets, sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice, c->stream));
    return XTN_SUCCESS;
}

static int stage_host(xtn_context* c, size_t bytes) {
    if (c->h_stage_cap >= bytes) return XTN_SUCCESS;
    if (c->h_stage) cudaFreeHost(c->h_stage);
    c->h_stage = nullptr;
    c->h_stage_cap = 0;
    size_t nb = bytes + bytes / 8 + 4096;
    XTN_CK(cudaMallocHost(&c->h_stage, nb));
    c->h_stage_cap = nb;
    return XTN_SUCCESS;
}

// Hands the device result to the callback in chunks of at most kChunk entries.
static int deliver(xtn_context* c, xtn_callback cb, void* user) {
    const int64_t kChunk = int64_t(1) << 24;
    int64_t n = c->n_out;
    if (!cb) return XTN_SUCCESS;
    int64_t chunk = std::min<int64_t>(std::max<int64_t>(n, 1), kChunk);
    size_t per = sizeof(xtn_int2) + (c->overlap_result ? sizeof(uint64_t) : 1);
    XTN_TRY(stage_host(c, per * chunk));
    xtn_int2* hp = reinterpret_cast<xtn_int2*>(c->h_stage);
    void* hv = reinterpret_cast<char*>(c->h_stage) + sizeof(xtn_int2) * chunk;
    if (n == 0) {
        xtn_output out{hp, c->overlap_result ? nullptr : reinterpret_cast<int8_t*>(hv),
                       c->overlap_result ? reinterpret_cast<uint64_t*>(hv) : nullptr, 0};
        cb(&out, user);
        return XTN_SUCCESS;
    }
    for (int64_t o = 0; o < n; o += chunk) {
        int64_t m = std::min(chunk, n - o);
        XTN_CK(cudaMemcpyAsync(hp, P<xtn_int2>(c->out_pairs) + o, sizeof(xtn_int2) * m, cudaMemcpyDeviceToHost, c->stream));
        if (c->overlap_result)
            XTN_CK(cudaMemcpyAsync(hv, P<uint64_t>(c->out_freq) + o, sizeof(uint64_t) * m, cudaMemcpyDeviceToHost,
                                   c->stream));
        else
            XTN_CK(cudaMemcpyAsync(hv, P<int8_t>(c->out_dist) + o, (size_t)m, cudaMemcpyDeviceToHost, c->stream));
        XTN_CK(cudaStreamSynchronize(c->stream));
        xtn_output out{hp, c->overlap_result ? nullptr : reinterpret_cast<int8_t*>(hv),
                       c->overlap_result ? reinterpret_cast<uint64_t*>(hv) : nullptr, m};
        cb(&out, user);
    }
    return XTN_SUCCESS;
}

// ------------------------------------------------------------------ overlap mode
// Repertoire overlap (S/src/xtn_overlap_inner.cu:57-245, S/src/kernel.cu:405-435,565-584):
//   1. rows with identical full strings are merged (hash sort + exact string check); the
//      occurrences of a unique string keep row order, as the reference's stable sort does;
//   2. diagonal term: for occurrences a <= b of one unique string, f_a*f_b is added to
//      (rep_a, rep_b);
//   3. the nearest-neighbour pipeline runs on one representative row per unique string;
//   4. cross term: for a verified unique pair (u, v) and occurrences a of u, b of v,
//      f_a*f_b (x2 when rep_a == rep_b) is added to (min rep, max rep);
//   5. the R x R matrix of sums (u64, wrapping like the reference's size_t) is emitted in
//      (x, y) order for every entry that received a contribution.

// Kernels of the overlap form take an abort word (nullptr in the plain form): the graph form
// sets it when the lengths or repertoire ids are invalid, or the unique-string count differs from
// the one the graph was captured for, and every kernel that would index by them then does nothing.
__device__ __forceinline__ bool aborted(const unsigned int* abort) { return abort && *abort; }

__global__ void k_row_hash(const uint8_t* __restrict__ chars, const uint32_t* __restrict__ offs, int n, int idbits,
                           uint64_t* __restrict__ recs, const unsigned int* __restrict__ abort) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || aborted(abort)) return;
    uint32_t s = offs[i];
    int L = (int)(offs[i + 1] - s);
    uint64_t h = 0x84222325cbf29ce4ULL ^ (uint64_t)L;
    for (int j = 0; j < L; j++) h = (h ^ chars[s + j]) * 0x100000001b3ULL;
    h = hash_fin(h);
    recs[i] = (h & ~((1ull << idbits) - 1ull)) | (uint64_t)i;
}

__device__ __forceinline__ int cmp_rows(const uint8_t* chars, const uint32_t* offs, uint32_t a, uint32_t b) {
    uint32_t sa = offs[a], sb = offs[b];
    int la = (int)(offs[a + 1] - sa), lb = (int)(offs[b + 1] - sb);
    int m = la < lb ? la : lb;
    for (int k = 0; k < m; k++) {
        int x = chars[sa + k], y = chars[sb + k];
        if (x != y) return x < y ? -1 : 1;
    }
    return la == lb ? 0 : (la < lb ? -1 : 1);
}

// A run of equal hashes that holds different strings (a hash collision) is re-ordered by
// (string, row) so that equal strings are contiguous again with rows ascending.
__global__ void k_run_fix(uint64_t* __restrict__ recs, int n, int idbits, const uint8_t* __restrict__ chars,
                          const uint32_t* __restrict__ offs, const unsigned int* __restrict__ abort) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || aborted(abort)) return;
    const uint64_t idmask = (1ull << idbits) - 1ull;
    uint64_t k = recs[i] >> idbits;
    if (i > 0 && (recs[i - 1] >> idbits) == k) return;
    int j = i + 1;
    bool mixed = false;
    while (j < n && (recs[j] >> idbits) == k) {
        if (cmp_rows(chars, offs, (uint32_t)(recs[i] & idmask), (uint32_t)(recs[j] & idmask)) != 0) mixed = true;
        j++;
    }
    if (!mixed) return;
    for (int a = i + 1; a < j; a++) {
        uint64_t v = recs[a];
        int b = a - 1;
        while (b >= i) {
            int c = cmp_rows(chars, offs, (uint32_t)(recs[b] & idmask), (uint32_t)(v & idmask));
            if (c < 0 || (c == 0 && (recs[b] & idmask) < (v & idmask))) break;
            recs[b + 1] = recs[b];
            b--;
        }
        recs[b + 1] = v;
    }
}

__global__ void k_uniq_flags(const uint64_t* __restrict__ recs, int n, int idbits, const uint8_t* __restrict__ chars,
                             const uint32_t* __restrict__ offs, uint8_t* __restrict__ head,
                             const unsigned int* __restrict__ abort) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (aborted(abort)) {
        head[i] = 0;
        return;
    }
    const uint64_t idmask = (1ull << idbits) - 1ull;
    bool h = i == 0 || (recs[i] >> idbits) != (recs[i - 1] >> idbits) ||
             cmp_rows(chars, offs, (uint32_t)(recs[i - 1] & idmask), (uint32_t)(recs[i] & idmask)) != 0;
    head[i] = h ? 1 : 0;
}

__global__ void k_uniq_build(const uint64_t* __restrict__ recs, const uint8_t* __restrict__ head,
                             const uint32_t* __restrict__ uidx, int n, int idbits, int32_t* __restrict__ rep_row,
                             uint32_t* __restrict__ occ_start, uint32_t* __restrict__ srow,
                             const unsigned int* __restrict__ abort) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || aborted(abort)) return;
    uint32_t row = (uint32_t)(recs[i] & ((1ull << idbits) - 1ull));
    srow[i] = row;
    if (head[i]) {
        uint32_t u = uidx[i];
        occ_start[u] = (uint32_t)i;
        rep_row[u] = (int32_t)row;
    }
    if (i == n - 1) occ_start[uidx[n]] = (uint32_t)n;
}

// Unique strings renumbered in row order (the order of their first occurrence), so that the
// search over them reads the character store in order: row_head[row] marks first occurrences;
// after an exclusive scan row_uid[row] is the row-order number of a first occurrence, and
// k_uniq_row_order fills row_rep (row-order number -> row, ascending) and row_map (row-order
// number -> hash-order number, which indexes the occurrence lists).
__global__ void k_uniq_row_heads(const int32_t* __restrict__ rep_row, int U, uint8_t* __restrict__ row_head,
                                 const unsigned int* __restrict__ abort) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < U && !aborted(abort)) row_head[rep_row[u]] = 1;
}

__global__ void k_uniq_row_order(const int32_t* __restrict__ rep_row, int U, const uint32_t* __restrict__ row_uid,
                                 int32_t* __restrict__ row_rep, uint32_t* __restrict__ row_map,
                                 const unsigned int* __restrict__ abort) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= U || aborted(abort)) return;
    const int32_t row = rep_row[u];
    const uint32_t v = row_uid[row];
    row_rep[v] = row;
    row_map[v] = (uint32_t)u;
}

__device__ __forceinline__ uint64_t freq_product(int32_t a, int32_t b) {
    return (uint64_t)(int64_t)a * (uint64_t)(int64_t)b;
}

// Diagonal term; with R <= kSmemReps the block accumulates into shared memory first.
constexpr int kSmemReps = 96;

__global__ void k_diag(const uint32_t* __restrict__ occ_start, const uint32_t* __restrict__ srow, int U,
                       const int32_t* __restrict__ freq, const int32_t* __restrict__ rep, int R,
                       unsigned long long* __restrict__ M, uint8_t* __restrict__ present,
                       const unsigned int* __restrict__ abort) {
    extern __shared__ unsigned long long s_m[];
    if (aborted(abort)) return;
    const bool local = R <= kSmemReps;
    uint8_t* s_p = reinterpret_cast<uint8_t*>(s_m + (local ? R * R : 0));
    if (local) {
        for (int k = threadIdx.x; k < R * R; k += blockDim.x) {
            s_m[k] = 0;
            s_p[k] = 0;
        }
        __syncthreads();
    }
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < U; u += gridDim.x * blockDim.x) {
        const uint32_t s = occ_start[u], e = occ_start[u + 1];
        for (uint32_t a = s; a < e; a++) {
            const uint32_t ra = srow[a];
            const int qa = rep[ra];
            const int32_t fa = freq[ra];
            for (uint32_t b = a; b < e; b++) {
                const uint32_t rb = srow[b];
                const size_t cell = (size_t)qa * R + rep[rb];
                const unsigned long long f = (unsigned long long)freq_product(fa, freq[rb]);
                if (local) {
                    atomicAdd(&s_m[cell], f);
                    s_p[cell] = 1;
                } else {
                    atomicAdd(&M[cell], f);
                    present[cell] = 1;
                }
            }
        }
    }
    if (local) {
        __syncthreads();
        for (int k = threadIdx.x; k < R * R; k += blockDim.x)
            if (s_p[k]) {
                atomicAdd(&M[k], s_m[k]);
                present[k] = 1;
            }
    }
}

// Cross term; with R <= kSmemReps the block accumulates into shared memory first. The graph
// form passes the verified-pair count on the device (np_dev) instead of np.
__global__ void k_cross(const xtn_int2* __restrict__ pairs, int64_t np, const uint32_t* __restrict__ occ_start,
                        const uint32_t* __restrict__ srow, const int32_t* __restrict__ freq,
                        const int32_t* __restrict__ rep, int R, unsigned long long* __restrict__ M,
                        uint8_t* __restrict__ present, const uint32_t* __restrict__ row_map,
                        const uint64_t* __restrict__ np_dev, const unsigned int* __restrict__ abort) {
    extern __shared__ unsigned long long s_m[];
    if (aborted(abort)) return;
    if (np_dev) np = (int64_t)*np_dev;
    const bool local = R <= kSmemReps;
    uint8_t* s_p = reinterpret_cast<uint8_t*>(s_m + (local ? R * R : 0));
    if (local) {
        for (int k = threadIdx.x; k < R * R; k += blockDim.x) {
            s_m[k] = 0;
            s_p[k] = 0;
        }
        __syncthreads();
    }
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < np; t += (int64_t)gridDim.x * blockDim.x) {
        const xtn_int2 pr = pairs[t];
        const uint32_t ux = row_map[pr.x], uy = row_map[pr.y];  // row-order -> hash-order numbers
        uint32_t s1 = occ_start[ux], e1 = occ_start[ux + 1];
        uint32_t s2 = occ_start[uy], e2 = occ_start[uy + 1];
        for (uint32_t a = s1; a < e1; a++) {
            uint32_t ra = srow[a];
            int qa = rep[ra];
            int32_t fa = freq[ra];
            for (uint32_t b = s2; b < e2; b++) {
                uint32_t rb = srow[b];
                int qb = rep[rb];
                uint64_t f = freq_product(fa, freq[rb]);
                if (qa == qb) f *= 2;
                int x = qa < qb ? qa : qb, y = qa < qb ? qb : qa;
                size_t cell = (size_t)x * R + y;
                if (local) {
                    atomicAdd(&s_m[cell], (unsigned long long)f);
                    s_p[cell] = 1;
                } else {
                    atomicAdd(&M[cell], (unsigned long long)f);
                    present[cell] = 1;
                }
            }
        }
    }
    if (local) {
        __syncthreads();
        for (int k = threadIdx.x; k < R * R; k += blockDim.x)
            if (s_p[k]) {
                atomicAdd(&M[k], s_m[k]);
                present[k] = 1;
            }
    }
}

__global__ void k_matrix_compact(const unsigned long long* __restrict__ M, const uint8_t* __restrict__ present,
                                 const uint32_t* __restrict__ pos, int R, xtn_int2* __restrict__ out,
                                 uint64_t* __restrict__ out_freq) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)R * R || !present[k]) return;
    uint32_t o = pos[k];
    out[o] = xtn_int2{(int32_t)(k / R), (int32_t)(k % R)};
    out_freq[o] = M[k];
}

}  // namespace xtn

struct xtn_overlap_bufs {
    DevBuf freq, rep, recA, recB, head, uidx, rep_row, occ_start, srow, M, present, mpos, scratch;
    DevBuf row_head, row_uid, row_rep, row_map;  // unique strings numbered in row order
};

namespace xtn {

constexpr int kMaxRepertoires = 8192;

static std::vector<DevBuf*> context_buffers(xtn_context* c) {
    std::vector<DevBuf*> v = {
        &c->chars,   &c->offs,      &c->keys,      &c->klen,     &c->vcnt,       &c->voff,     &c->recA,
        &c->recB,    &c->gstart,    &c->gsize,     &c->gcnt,     &c->goff,       &c->pairA,    &c->pairB,
        &c->dist,    &c->flag,      &c->fpos,      &c->scratch64, &c->scratch32, &c->counter,  &c->out_pairs,
        &c->out_dist, &c->out_freq, &c->bcounts,   &c->boffs,    &c->btotals,    &c->bstart,   &c->bdesc,
        &c->bjobs,   &c->bfall,     &c->bcnt,      &c->fbA,      &c->fbB,        &c->runinfo,  &c->tcnt,
        &c->toff,    &c->ktab,      &c->info,      &c->lencheck, &c->pairA2,     &c->ddcnt,    &c->tseq,
        &c->os_scratch, &c->os_status, &c->dev_err, &c->dd_table, &c->scan_status, &c->scur, &c->gruns};
    if (c->overlap_bufs) {
        xtn_overlap_bufs* ob = reinterpret_cast<xtn_overlap_bufs*>(c->overlap_bufs);
        for (DevBuf* b : {&ob->freq, &ob->rep, &ob->recA, &ob->recB, &ob->head, &ob->uidx, &ob->rep_row,
                          &ob->occ_start, &ob->srow, &ob->M, &ob->present, &ob->mpos, &ob->scratch, &ob->row_head,
                          &ob->row_uid, &ob->row_rep, &ob->row_map})
            v.push_back(b);
    }
    return v;
}

static std::vector<const void*> context_buffer_ptrs(const xtn_context* c) {
    std::vector<const void*> v;
    for (const DevBuf* b : context_buffers(const_cast<xtn_context*>(c))) v.push_back(b->p);
    return v;
}

// De-interleaves the per-row info into frequency and repertoire arrays; *bad_row receives the
// smallest row whose repertoire id is outside [0, R) (it starts at INT_MAX).
__global__ void k_split_info(const xtn_seq_info* __restrict__ info, int n, int R, int32_t* __restrict__ freq,
                             int32_t* __restrict__ rep, int* __restrict__ bad_row) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const xtn_seq_info v = info[i];
    freq[i] = v.frequency;
    rep[i] = v.repertoire;
    if (v.repertoire < 0 || v.repertoire >= R) atomicMin(bad_row, i);
}

// The overlap form's buffers: everything indexed by a unique string is sized for n + 1 entries
// (the unique count is at most n), so that no stage has to wait for that count to size them.
static int ov_reserve(xtn_context* c, xtn_overlap_bufs& b, int n, int R) {
    const size_t RR = (size_t)R * R;
    XTN_TRY(ensure(b.freq, sizeof(int32_t) * n));
    XTN_TRY(ensure(b.rep, sizeof(int32_t) * n));
    XTN_TRY(ensure(c->counter, 64));
    XTN_TRY(ensure(b.recA, sizeof(uint64_t) * n));
    XTN_TRY(ensure(b.recB, sizeof(uint64_t) * n));
    XTN_TRY(ensure(c->scratch32, sizeof(uint32_t) * radix_scratch_elems(n)));
    XTN_TRY(ensure(b.head, (size_t)n));
    XTN_TRY(ensure(b.uidx, sizeof(uint32_t) * (n + 1)));
    XTN_TRY(ensure(b.scratch, sizeof(uint32_t) * std::max(scan_scratch_elems(n), scan_scratch_elems((int64_t)RR))));
    XTN_TRY(ensure(b.rep_row, sizeof(int32_t) * (n + 1)));
    XTN_TRY(ensure(b.occ_start, sizeof(uint32_t) * (n + 1)));
    XTN_TRY(ensure(b.srow, sizeof(uint32_t) * n));
    XTN_TRY(ensure(b.row_head, (size_t)n));
    XTN_TRY(ensure(b.row_uid, sizeof(uint32_t) * (n + 1)));
    XTN_TRY(ensure(b.row_rep, sizeof(int32_t) * (n + 1)));
    XTN_TRY(ensure(b.row_map, sizeof(uint32_t) * (n + 1)));
    XTN_TRY(ensure(b.M, sizeof(unsigned long long) * RR));
    XTN_TRY(ensure(b.present, RR));
    XTN_TRY(ensure(b.mpos, sizeof(uint32_t) * (RR + 1)));
    XTN_TRY(ensure(c->scan_status, sizeof(unsigned long long) * scan_1p_words(n)));
    XTN_TRY(ensure_err_word(c));
    const size_t msmem = R <= kSmemReps ? RR * (sizeof(unsigned long long) + 1) : 0;
    if (msmem > 48 * 1024) {
        XTN_CK(cudaFuncSetAttribute(k_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem));
        XTN_CK(cudaFuncSetAttribute(k_cross, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem));
    }
    return XTN_SUCCESS;
}

static size_t ov_matrix_smem(int R) {
    return R <= kSmemReps ? (size_t)R * R * (sizeof(unsigned long long) + 1) : 0;
}

// 1. identical strings merged: row hashes sorted, hash collisions re-ordered by string, first
// occurrences flagged and numbered (uidx[n] = U), occurrence lists (occ_start, srow) and one
// representative row per unique string (rep_row, hash order).
static void ov_unique(xtn_context* c, xtn_overlap_bufs& b, const uint8_t* chars, const uint32_t* offs, int n,
                      const unsigned int* abort) {
    cudaStream_t s = c->stream;
    const int idbits = id_bits_for(n);
    XTN_LAUNCH("row_hash", k_row_hash<<<blocks_for(n), kThreads, 0, s>>>(chars, offs, n, idbits, P<uint64_t>(b.recA),
                                                                          abort));
    uint64_t* recs = radix_sort_u64(P<uint64_t>(b.recA), P<uint64_t>(b.recB), n, idbits, 64, P<uint32_t>(c->scratch32),
                                    s, "row_sort_upsweep", "row_sort_downsweep");
    XTN_LAUNCH("run_fix", k_run_fix<<<blocks_for(n), kThreads, 0, s>>>(recs, n, idbits, chars, offs, abort));
    XTN_LAUNCH("uniq_flags", k_uniq_flags<<<blocks_for(n), kThreads, 0, s>>>(recs, n, idbits, chars, offs,
                                                                              P<uint8_t>(b.head), abort));
    scan_exclusive<uint8_t, uint32_t>(P<uint8_t>(b.head), P<uint32_t>(b.uidx), n, P<uint32_t>(b.scratch), s);
    XTN_LAUNCH("uniq_build", k_uniq_build<<<blocks_for(n), kThreads, 0, s>>>(
                                 recs, P<uint8_t>(b.head), P<uint32_t>(b.uidx), n, idbits, P<int32_t>(b.rep_row),
                                 P<uint32_t>(b.occ_start), P<uint32_t>(b.srow), abort));
}

// The unique strings renumbered in row order (row_rep: row-order number -> row, row_map:
// row-order number -> hash-order number), then the diagonal term into the cleared matrix.
static int ov_rows_diag(xtn_context* c, xtn_overlap_bufs& b, int n, uint32_t U, int R, const unsigned int* abort) {
    cudaStream_t s = c->stream;
    const size_t RR = (size_t)R * R;
    XTN_CK(cudaMemsetAsync(b.row_head.p, 0, (size_t)n, s));
    XTN_LAUNCH("uniq_row_heads", k_uniq_row_heads<<<blocks_for((int64_t)U), kThreads, 0, s>>>(
                                     P<int32_t>(b.rep_row), (int)U, P<uint8_t>(b.row_head), abort));
    scan_exclusive_1p<uint8_t, uint32_t>(P<uint8_t>(b.row_head), P<uint32_t>(b.row_uid), n,
                                         P<unsigned long long>(c->scan_status), P<unsigned int>(c->dev_err), s,
                                         c->wait_polls, 0);
    XTN_LAUNCH("uniq_row_order", k_uniq_row_order<<<blocks_for((int64_t)U), kThreads, 0, s>>>(
                                     P<int32_t>(b.rep_row), (int)U, P<uint32_t>(b.row_uid), P<int32_t>(b.row_rep),
                                     P<uint32_t>(b.row_map), abort));
    XTN_CK(cudaMemsetAsync(b.M.p, 0, sizeof(unsigned long long) * RR, s));
    XTN_CK(cudaMemsetAsync(b.present.p, 0, RR, s));
    const unsigned dblocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(blocks_for((int64_t)U), c->sms * 4));
    XTN_LAUNCH("diag", k_diag<<<dblocks, kThreads, ov_matrix_smem(R), s>>>(
                           P<uint32_t>(b.occ_start), P<uint32_t>(b.srow), (int)U, P<int32_t>(b.freq), P<int32_t>(b.rep),
                           R, P<unsigned long long>(b.M), P<uint8_t>(b.present), abort));
    return XTN_SUCCESS;
}

// 4. cross term over the verified unique pairs (np on the host, or *np_dev on the device).
static void ov_cross(xtn_context* c, xtn_overlap_bufs& b, int64_t np, const uint64_t* np_dev, int R,
                     const unsigned int* abort) {
    const int64_t blocks = np_dev ? (int64_t)c->sms * 4 : std::min<int64_t>((np + kThreads - 1) / kThreads, (int64_t)c->sms * 4);
    XTN_LAUNCH("cross", k_cross<<<(unsigned)std::max<int64_t>(blocks, 1), kThreads, ov_matrix_smem(R), c->stream>>>(
                            P<xtn_int2>(c->out_pairs), np, P<uint32_t>(b.occ_start), P<uint32_t>(b.srow),
                            P<int32_t>(b.freq), P<int32_t>(b.rep), R, P<unsigned long long>(b.M),
                            P<uint8_t>(b.present), P<uint32_t>(b.row_map), np_dev, abort));
}

// 5. matrix -> entries in (x, y) order (positions scanned from the presence flags; the count is
// mpos[R * R]).
static void ov_matrix(xtn_context* c, xtn_overlap_bufs& b, int R, bool scan) {
    const size_t RR = (size_t)R * R;
    if (scan)
        scan_exclusive<uint8_t, uint32_t>(P<uint8_t>(b.present), P<uint32_t>(b.mpos), (int64_t)RR,
                                          P<uint32_t>(b.scratch), c->stream);
    else
        XTN_LAUNCH("matrix_compact", k_matrix_compact<<<blocks_for((int64_t)RR), kThreads, 0, c->stream>>>(
                                         P<unsigned long long>(b.M), P<uint8_t>(b.present), P<uint32_t>(b.mpos), R,
                                         P<xtn_int2>(c->out_pairs), P<uint64_t>(c->out_freq)));
}

// Overlap mode on device-resident inputs (d_info: one xtn_seq_info per row, row order).
int run_overlap(xtn_context* c, const uint8_t* chars, const uint32_t* offs, const xtn_seq_info* d_info, int n, int d,
                int measure, int R, bool validate) {
    if (c->shard_count > 1) {
        set_err("sharding covers the nearest-neighbour mode only");
        return XTN_ERR_ARG;
    }
    if (R > kMaxRepertoires) {
        set_err("overlap mode supports at most " + std::to_string(kMaxRepertoires) + " repertoires");
        return XTN_ERR_LIMIT;
    }
    cudaStream_t s = c->stream;
    xtn_overlap_bufs& b = *reinterpret_cast<xtn_overlap_bufs*>(c->overlap_bufs);
    XTN_TRY(ov_reserve(c, b, n, R));
    const int int_max = 0x7fffffff;
    XTN_CK(cudaMemcpyAsync(c->counter.p, &int_max, sizeof(int), cudaMemcpyHostToDevice, s));
    if (validate) XTN_TRY(launch_length_check(c, offs, nullptr, n));
    XTN_LAUNCH("split_info", k_split_info<<<blocks_for(n), kThreads, 0, s>>>(d_info, n, R, P<int32_t>(b.freq),
                                                                              P<int32_t>(b.rep), P<int>(c->counter)));
    XTN_CK(cudaGetLastError());
    uint64_t bad = 0;
    if (validate) XTN_CK(cudaMemcpyAsync(c->h_scalar + 1, c->lencheck.p, 4, cudaMemcpyDeviceToHost, s));
    XTN_TRY(read_scalar(c, c->counter.p, 4, &bad));
    if (validate) XTN_TRY(length_check_result(c, (uint32_t)c->h_scalar[1]));
    if ((int)bad != int_max) {
        set_err("repertoire id out of range at row " + std::to_string((int)bad));
        return XTN_ERR_ARG;
    }

    // 1. merge identical strings
    ov_unique(c, b, chars, offs, n, nullptr);
    XTN_CK(cudaGetLastError());
    uint64_t U = 0;
    XTN_TRY(read_scalar(c, P<uint32_t>(b.uidx) + n, 4, &U));
    // 2. row-order numbering, diagonal term
    XTN_TRY(ov_rows_diag(c, b, n, (uint32_t)U, R, nullptr));
    XTN_CK(cudaGetLastError());

    // 3. neighbours among the unique strings
    XTN_TRY(run_nn(c, chars, offs, P<int32_t>(b.row_rep), (int)U, d, measure, false));
    const int64_t nverified = c->n_out;

    // 4. cross term
    if (nverified > 0) ov_cross(c, b, nverified, nullptr, R, nullptr);
    XTN_CK(cudaGetLastError());

    // 5. matrix -> sorted entries
    const size_t RR = (size_t)R * R;
    ov_matrix(c, b, R, true);
    uint64_t nent = 0;
    XTN_TRY(read_scalar(c, P<uint32_t>(b.mpos) + RR, 4, &nent));
    XTN_TRY(ensure(c->out_pairs, sizeof(xtn_int2) * nent));
    XTN_TRY(ensure(c->out_freq, sizeof(uint64_t) * nent));
    ov_matrix(c, b, R, false);
    XTN_CK(cudaGetLastError());
    XTN_CK(cudaStreamSynchronize(s));
    c->n_out = (int64_t)nent;
    c->overlap_result = true;
    c->stats.n_verified_pairs = nverified;
    c->stats.n_out = (int64_t)nent;
    c->stats.n_seqs = (int64_t)U;
    return XTN_SUCCESS;
}

// ------------------------------------------------------------------ overlap graph form
// The overlap mode on device-resident inputs as one captured launch sequence (option "graph"):
// the length and repertoire checks, the merge of identical strings, the row-order numbering and
// the diagonal term, the whole neighbour search over the unique strings as the search's graph
// form enqueues it (persistent grouping, device-side sizes), the cross term over the verified
// count on the device and the matrix compaction, with one status block read per replay. The
// unique-string count and the search's capacities come from the plain run that precedes the
// capture; a replay whose unique count differs, or whose search outgrows a capacity, is redone
// by the plain form, which re-captures.
struct OverlapGraph {
    const uint8_t* chars = nullptr;
    const uint32_t* offs = nullptr;
    const xtn_seq_info* info = nullptr;
    int n = 0, d = 0, measure = 0, R = 0;
    GraphSig sig{};
    uint32_t U = 0;
    GraphState nn;  // capacities and device tables of the search over the unique strings
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;
    std::vector<const void*> bufs;  // the context's buffers at capture (a reallocation invalidates it)
    DevBuf ost;  // u32 [0] first bad repertoire row, [1] first bad length, [2] abort word
};

// Overlap status words, copied to the pinned host scalars 29..31.
enum { OS_BAD, OS_UNIQUE, OS_ENTRIES, OS_WORDS };

__global__ void k_overlap_guard(const unsigned int* __restrict__ ost, unsigned int* __restrict__ abort) {
    abort[0] = (ost[0] != 0x7fffffffu || ost[1] != 0xffffffffu) ? 1u : 0u;
}

__global__ void k_overlap_unique_guard(const uint32_t* __restrict__ U_dev, uint32_t U, unsigned int* __restrict__ abort) {
    if (*U_dev != U) abort[0] = 1u;
}

__global__ void k_overlap_status(const unsigned int* __restrict__ ost, const uint32_t* __restrict__ U_dev,
                                 const uint32_t* __restrict__ nent, uint64_t* __restrict__ st) {
    st[OS_BAD] = (uint64_t)ost[0] | ((uint64_t)ost[1] << 32);
    st[OS_UNIQUE] = *U_dev;
    st[OS_ENTRIES] = *nent;
}

static void overlap_graph_release(OverlapGraph* og) {
    if (og->exec) cudaGraphExecDestroy(og->exec);
    if (og->graph) cudaGraphDestroy(og->graph);
    og->exec = nullptr;
    og->graph = nullptr;
}

static int overlap_graph_enqueue(xtn_context* c, OverlapGraph* og) {
    cudaStream_t s = c->stream;
    xtn_overlap_bufs& b = *reinterpret_cast<xtn_overlap_bufs*>(c->overlap_bufs);
    const int n = og->n, R = og->R;
    unsigned int* ost = P<unsigned int>(og->ost);
    unsigned int* abort = ost + 2;
    XTN_LAUNCH("set_status", k_set_u64<<<1, 1, 0, s>>>(reinterpret_cast<unsigned long long*>(ost),
                                                       0xffffffff7fffffffull));
    XTN_LAUNCH("check_lengths", k_check_lengths<<<blocks_for(n), kThreads, 0, s>>>(og->offs, nullptr, n, ost + 1));
    XTN_LAUNCH("split_info", k_split_info<<<blocks_for(n), kThreads, 0, s>>>(og->info, n, R, P<int32_t>(b.freq),
                                                                              P<int32_t>(b.rep), reinterpret_cast<int*>(ost)));
    XTN_LAUNCH("overlap_guard", k_overlap_guard<<<1, 1, 0, s>>>(ost, abort));
    ov_unique(c, b, og->chars, og->offs, n, abort);
    XTN_LAUNCH("overlap_guard", k_overlap_unique_guard<<<1, 1, 0, s>>>(P<uint32_t>(b.uidx) + n, og->U, abort));
    // rows the search reads when an abort leaves them unset
    XTN_CK(cudaMemsetAsync(b.row_rep.p, 0, sizeof(int32_t) * (og->U + 1), s));
    XTN_TRY(ov_rows_diag(c, b, n, og->U, R, abort));
    og->nn.rows = P<int32_t>(b.row_rep);
    og->nn.pre_abort = abort;
    XTN_TRY(graph_enqueue(c, &og->nn));
    ov_cross(c, b, 0, P<uint64_t>(og->nn.status) + GS_OUT, R, abort);
    ov_matrix(c, b, R, true);
    ov_matrix(c, b, R, false);
    XTN_LAUNCH("overlap_status", k_overlap_status<<<1, 1, 0, s>>>(ost, P<uint32_t>(b.uidx) + n,
                                                                   P<uint32_t>(b.mpos) + (size_t)R * R,
                                                                   P<uint64_t>(og->ost) + 2));
    XTN_CK(cudaMemcpyAsync(c->h_scalar + 29, P<uint64_t>(og->ost) + 2, sizeof(uint64_t) * OS_WORDS,
                           cudaMemcpyDeviceToHost, s));
    XTN_CK(cudaGetLastError());
    return XTN_SUCCESS;
}

// Capacities from the plain overlap run just made on this input, buffers reserved, graph captured.
static int overlap_graph_build(xtn_context* c, OverlapGraph* og, const uint8_t* chars, const uint32_t* offs,
                               const xtn_seq_info* info, int n, int d, int measure, int R) {
    overlap_graph_release(og);
    xtn_overlap_bufs& b = *reinterpret_cast<xtn_overlap_bufs*>(c->overlap_bufs);
    const uint32_t U = (uint32_t)c->stats.n_seqs;
    const size_t RR = (size_t)R * R;
    if (RR > ((size_t)1 << 24)) return XTN_ERR_LIMIT;  // matrix output capacity: at most 2^24 entries
    og->chars = chars;
    og->offs = offs;
    og->info = info;
    og->n = n;
    og->d = d;
    og->measure = measure;
    og->R = R;
    og->U = U;
    og->sig = graph_signature(c);
    XTN_TRY(graph_reserve(c, &og->nn, chars, offs, P<int32_t>(b.row_rep), (int)U, d, measure));
    XTN_TRY(ov_reserve(c, b, n, R));
    // the matrix entries of the plain run are still to be read by the caller
    XTN_TRY(ensure_keep(c, c->out_pairs, std::max<size_t>(c->out_pairs.cap, sizeof(xtn_int2) * RR + 64),
                        sizeof(xtn_int2) * (size_t)c->n_out));
    XTN_TRY(ensure_keep(c, c->out_freq, sizeof(uint64_t) * RR + 64, sizeof(uint64_t) * (size_t)c->n_out));
    XTN_TRY(ensure(og->ost, 64));
    XTN_CK(cudaStreamSynchronize(c->stream));
    cudaGraph_t graph = nullptr;
    XTN_TRY(capture(c, [&] { return overlap_graph_enqueue(c, og); }, &graph, &og->launches));
    og->graph = graph;
    XTN_CK(cudaGraphInstantiate(&og->exec, graph, 0));
    og->bufs = context_buffer_ptrs(c);
    return XTN_SUCCESS;
}

static int overlap_graph_replay(xtn_context* c, OverlapGraph* og, bool* redo) {
    *redo = false;
    XTN_TRY(graph_launch(c, og->exec));
    xtn_stats& st = c->stats;
    const uint64_t* h = c->h_scalar + 29;
    const uint32_t lenbad = (uint32_t)(h[OS_BAD] >> 32);
    const int bad = (int)(uint32_t)h[OS_BAD];
    if (lenbad != 0xffffffffu) return length_check_result(c, lenbad);
    if (bad != 0x7fffffff) {
        set_err("repertoire id out of range at row " + std::to_string(bad));
        return XTN_ERR_ARG;
    }
    if (h[OS_UNIQUE] != og->U) {
        *redo = true;
        return XTN_SUCCESS;
    }
    const float ms = st.ms_total;
    XTN_TRY(graph_check(c, &og->nn, redo));
    if (*redo) return XTN_SUCCESS;
    st.ms_total = ms;
    st.n_launches = og->launches;
    st.n_verified_pairs = st.n_out;
    st.n_out = (int64_t)h[OS_ENTRIES];
    st.n_seqs = (int64_t)og->U;
    c->n_out = st.n_out;
    c->overlap_result = true;
    return XTN_SUCCESS;
}

// The device-resident overlap mode in the graph form (option "graph" = 1).
static int overlap_graph(xtn_context* c, const uint8_t* chars, const uint32_t* offs, const xtn_seq_info* info, int n,
                         int d, int measure, int R) {
    if (!c->ograph) c->ograph = new OverlapGraph();
    OverlapGraph* og = static_cast<OverlapGraph*>(c->ograph);
    const bool same = og->exec && og->chars == chars && og->offs == offs && og->info == info && og->n == n &&
                      og->d == d && og->measure == measure && og->R == R && og->sig == graph_signature(c) &&
                      og->bufs == context_buffer_ptrs(c);
    if (same) {
        bool redo = false;
        XTN_TRY(overlap_graph_replay(c, og, &redo));
        if (!redo) return XTN_SUCCESS;
    }
    begin_run(c);
    int r = run_overlap(c, chars, offs, info, n, d, measure, R, true);
    end_run(c);
    if (r != XTN_SUCCESS) return r;
    const xtn_stats keep = c->stats;
    const int64_t keep_out = c->n_out;
    const int b = overlap_graph_build(c, og, chars, offs, info, n, d, measure, R);
    if (b != XTN_SUCCESS && b != XTN_ERR_LIMIT) return b;
    if (b == XTN_ERR_LIMIT) overlap_graph_release(og);  // this input stays in the plain form
    c->stats = keep;
    c->n_out = keep_out;
    c->overlap_result = true;
    return XTN_SUCCESS;
}

}  // namespace xtn

namespace xtn {
// ------------------------------------------------------------------ autotuner
// The shape of a search - first-level and split stage chunks, first-level bucket bits, bulk-copy
// or plain loads in the grouping kernel, the verification variant, and the plain or graph
// form - chosen by timing on the caller's device-resident data, and remembered per input class:
// the size (log2 n), distance, measure, the median sequence length and the share of sequences
// longer than the 18-residue key (whose pairs take the long verification path). The reference's
// sizes are fixed (xtneighbor_streaming/src/xtn.cu:21-26).
struct TuneShape {
    int stage, split, bits, tma, verify, graph, flat;
};
struct TuneKey {
    int log2n, d, measure, len_med, long_share;  // long_share in percent
    bool operator==(const TuneKey& o) const {
        return log2n == o.log2n && d == o.d && measure == o.measure && len_med == o.len_med &&
               long_share == o.long_share;
    }
};
struct TuneCache {
    std::vector<std::pair<TuneKey, TuneShape>> entries;
};

constexpr int kLenBins = 34;  // lengths 0..32, then longer

__global__ void k_len_hist(const uint32_t* __restrict__ offs, int n, unsigned int* __restrict__ hist) {
    __shared__ unsigned int h[kLenBins];
    for (int i = threadIdx.x; i < kLenBins; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t L = offs[i + 1] - offs[i];
        atomicAdd(&h[L < (uint32_t)kLenBins - 1 ? L : kLenBins - 1], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kLenBins; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

static int tune_key(xtn_context* c, const uint32_t* offs, int n, int d, int measure, TuneKey* key) {
    XTN_TRY(ensure(c->scratch64, sizeof(unsigned int) * kLenBins));
    XTN_CK(cudaMemsetAsync(c->scratch64.p, 0, sizeof(unsigned int) * kLenBins, c->stream));
    XTN_LAUNCH("len_hist", k_len_hist<<<std::max(1, std::min<int>((n + kThreads - 1) / kThreads, c->sms * 4)), kThreads,
                                        0, c->stream>>>(offs, n, P<unsigned int>(c->scratch64)));
    unsigned int h[kLenBins];
    XTN_CK(cudaMemcpyAsync(h, c->scratch64.p, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    XTN_CK(cudaStreamSynchronize(c->stream));
    int64_t acc = 0, longer = 0;
    int med = 0;
    for (int b = 0; b < kLenBins; b++) {
        if (acc * 2 < n) med = b;
        acc += h[b];
        if (b > kKeyLen) longer += h[b];
    }
    key->log2n = id_bits_for(n);
    key->d = d;
    key->measure = measure;
    key->len_med = med;
    key->long_share = (int)(100 * longer / std::max(1, n));
    return XTN_SUCCESS;
}

static void tune_apply(xtn_context* c, const TuneShape& sh) {
    c->stage_chunk = sh.stage;
    c->split_chunk = sh.split;
    c->bucket_bits_max = sh.bits;
    c->group_tma = sh.tma;
    c->verify_per = sh.verify;
    c->graph_mode = sh.graph;
    c->flat_gen = sh.flat;
}

static int nn_graph(xtn_context* c, const uint8_t* chars, const uint32_t* offs, int n, int d, int measure);

// One search as the context's shape says (plain or graph form).
static int tuned_search(xtn_context* c, const uint8_t* chars, const uint32_t* offs, int n, int d, int measure) {
    if (c->graph_mode) return nn_graph(c, chars, offs, n, d, measure);
    begin_run(c);
    const int r = run_nn(c, chars, offs, nullptr, n, d, measure, true);
    end_run(c);
    return r;
}

static int autotune(xtn_context* c, const xtn_args* args, const uint8_t* chars, const uint32_t* offs, int n,
                    int repeats, char* report, int report_cap) {
    if (repeats < 1) repeats = 2;
    const int d = args->distance, measure = args->measure;
    TuneKey key{};
    XTN_TRY(tune_key(c, offs, n, d, measure, &key));
    const TuneShape saved{c->stage_chunk, c->split_chunk, c->bucket_bits_max, c->group_tma,
                          c->verify_per,  c->graph_mode,  c->flat_gen};
    const int saved_engine = c->engine;
    c->engine = 0;
    auto time_shape = [&](const TuneShape& sh, float* ms) -> int {
        tune_apply(c, sh);
        float best = 1e30f;
        for (int r = 0; r <= repeats + sh.graph; r++) {  // warm-up first (the graph form: plain + capture too)
            const int st = tuned_search(c, chars, offs, n, d, measure);
            if (st != XTN_SUCCESS) return st;
            if (r > sh.graph) best = std::min(best, (float)c->stats.ms_total);
        }
        *ms = best;
        return XTN_SUCCESS;
    };
    TuneShape best{4096, 0, kMaxFirstLevelBits, 1, 1, 0, 1};
    float best_ms = 1e30f;
    int tried = 0;
    auto consider = [&](const TuneShape& sh) -> int {
        float ms = 0;
        const int st = time_shape(sh, &ms);
        if (st != XTN_SUCCESS) return st;
        tried++;
        if (ms < best_ms) {
            best_ms = ms;
            best = sh;
        }
        return XTN_SUCCESS;
    };
    int st = XTN_SUCCESS;
    // first level (generate-then-partition, or the one-pass scatter in two stage shapes), split
    // stage shape and first-level bits
    for (int flat : {1, 0})
        for (int stage : {4096, 2048})
            for (int split : {0, 2048})
                for (int bits : {9, 10}) {
                    if (st != XTN_SUCCESS) break;
                    if (bits == 10 && stage == 2048) continue;  // 1024 first-level buckets need the large shape
                    if (flat && stage != 4096) continue;         // the two-pass first level has one shape
                    st = consider(TuneShape{stage, split, bits, 1, 1, 0, flat});
                }
    // then, one at a time on the best so far: plain loads in grouping, the verification
    // variants, the graph form
    if (st == XTN_SUCCESS) {
        TuneShape sh = best;
        sh.tma = 0;
        st = consider(sh);
    }
    for (int per : {4, 8}) {
        if (st != XTN_SUCCESS) break;
        TuneShape sh = best;
        sh.verify = per;
        st = consider(sh);
    }
    if (st == XTN_SUCCESS) {
        TuneShape sh = best;
        sh.graph = 1;
        st = consider(sh);
    }
    c->engine = saved_engine;
    if (st != XTN_SUCCESS) {
        tune_apply(c, saved);
        return st;
    }
    tune_apply(c, best);
    if (!c->tune_cache) c->tune_cache = new TuneCache();
    TuneCache* tc = static_cast<TuneCache*>(c->tune_cache);
    bool stored = false;
    for (auto& e : tc->entries)
        if (e.first == key) {
            e.second = best;
            stored = true;
        }
    if (!stored) tc->entries.push_back({key, best});
    if (report && report_cap > 0)
        snprintf(report, (size_t)report_cap,
                 "flat_gen=%d stage_chunk=%d split_chunk=%d bucket_bits_max=%d group_tma=%d verify_per=%d graph=%d: "
                 "%.3f ms (best of %d shapes; input class log2n=%d d=%d measure=%d median_len=%d longer_than_key=%d%%)",
                 best.flat, best.stage, best.split, best.bits, best.tma, best.verify, best.graph, best_ms, tried, key.log2n,
                 key.d, key.measure, key.len_med, key.long_share);
    return XTN_SUCCESS;
}

// Option autotune = 1: the shape for this input's class comes from the cache, or is tuned now.
static int autotune_lookup(xtn_context* c, const xtn_args* args, const uint8_t* chars, const uint32_t* offs, int n) {
    TuneKey key{};
    XTN_TRY(tune_key(c, offs, n, args->distance, args->measure, &key));
    if (c->tune_cache)
        for (const auto& e : static_cast<TuneCache*>(c->tune_cache)->entries)
            if (e.first == key) {
                tune_apply(c, e.second);
                return XTN_SUCCESS;
            }
    return autotune(c, args, chars, offs, n, 2, nullptr, 0);
}

}  // namespace xtn

// ------------------------------------------------------------------ C ABI
extern "C" {

const char* xtn_last_error(void) { return t_err.c_str(); }

const char* xtn_version(void) { return "2.0.0 (xtn_b200 sm_100a)"; }

int xtn_context_create(int device, xtn_context** out) {
    if (!out) {
        set_err("null output pointer");
        return XTN_ERR_ARG;
    }
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_err(std::string("no CUDA device: ") + cudaGetErrorString(e));
        return XTN_ERR_NODEV;
    }
    if (device < 0 || device >= ndev) {
        set_err("device index out of range");
        return XTN_ERR_ARG;
    }
    XTN_CK(cudaSetDevice(device));
    xtn_context* c = new xtn_context();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost(&c->h_scalar, 256) != cudaSuccess) {
        set_err("stream or pinned scalar allocation failed");
        delete c;
        return XTN_ERR_CUDA;
    }
    for (auto& ev : c->ev) cudaEventCreate(&ev);
    for (auto& ev : c->ev_round) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    {
        size_t free_b = 0;
        cudaMemGetInfo(&free_b, &c->total_mem);
    }
    c->overlap_bufs = new xtn_overlap_bufs();
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    if (const char* e = getenv("XTN_ENGINE")) c->engine = (strcmp(e, "sort") == 0) ? 1 : 0;
    *out = c;
    return XTN_SUCCESS;
}

void xtn_context_destroy(xtn_context* c) {
    if (!c) return;
    if (current_profiler() == &c->prof) current_profiler() = nullptr;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->graph) {
        GraphState* g = static_cast<GraphState*>(c->graph);
        graph_release(g);
        release(g->status);
        release(g->table);
        release(g->os_status);
        delete g;
    }
    if (c->ograph) {
        OverlapGraph* og = static_cast<OverlapGraph*>(c->ograph);
        overlap_graph_release(og);
        release(og->nn.status);
        release(og->nn.table);
        release(og->nn.os_status);
        release(og->ost);
        delete og;
    }
    for (DevBuf* b : context_buffers(c)) release(*b);
    delete static_cast<TuneCache*>(c->tune_cache);
    delete reinterpret_cast<xtn_overlap_bufs*>(c->overlap_bufs);
    for (auto& ev : c->ev)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : c->ev_round)
        if (ev) cudaEventDestroy(ev);
    if (c->stream2) {
        cudaStreamSynchronize(c->stream2);
        cudaStreamDestroy(c->stream2);
    }
    if (c->h_scalar) cudaFreeHost(c->h_scalar);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

void* xtn_context_stream(xtn_context* c) { return c ? (void*)c->stream : nullptr; }

int xtn_context_stats(const xtn_context* c, xtn_stats* out) {
    if (!c || !out) return XTN_ERR_ARG;
    *out = c->stats;
    return XTN_SUCCESS;
}

int xtn_context_nn_device(xtn_context* c, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                          int32_t n, int64_t* n_out) {
    if (!c || !d_seqs || !d_offsets || n < 1) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    XTN_TRY(check_args(args));
    XTN_CK(cudaSetDevice(c->device));
    if (c->autotune_auto)
        XTN_TRY(autotune_lookup(c, args, reinterpret_cast<const uint8_t*>(d_seqs), d_offsets, n));
    int r;
    if (c->graph_mode) {
        r = nn_graph(c, reinterpret_cast<const uint8_t*>(d_seqs), d_offsets, n, args->distance, args->measure);
    } else {
        begin_run(c);
        r = run_nn(c, reinterpret_cast<const uint8_t*>(d_seqs), d_offsets, nullptr, n, args->distance, args->measure,
                   true);
        end_run(c);
    }
    if (r == XTN_SUCCESS && n_out) *n_out = c->n_out;
    return r;
}

int xtn_context_overlap_device(xtn_context* c, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                               int32_t n, const xtn_seq_info* d_info, int64_t* n_out) {
    if (!c || !d_seqs || !d_offsets || !d_info || n < 1) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    XTN_TRY(check_args(args));
    if (args->info_len < 1) {
        set_err("invalid info length");
        return XTN_ERR_ARG;
    }
    XTN_CK(cudaSetDevice(c->device));
    int r;
    if (c->graph_mode) {
        r = overlap_graph(c, reinterpret_cast<const uint8_t*>(d_seqs), d_offsets, d_info, n, args->distance,
                          args->measure, args->info_len);
    } else {
        begin_run(c);
        r = run_overlap(c, reinterpret_cast<const uint8_t*>(d_seqs), d_offsets, d_info, n, args->distance,
                        args->measure, args->info_len, true);
        end_run(c);
    }
    if (r == XTN_SUCCESS && n_out) *n_out = c->n_out;
    return r;
}

int xtn_context_perform(xtn_context* c, const xtn_args* args, const char* seqs, const uint32_t* offsets, int32_t n,
                        const xtn_seq_info* info, xtn_callback cb, void* user) {
    if (!c || !seqs || !offsets || n < 1) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    XTN_TRY(check_args(args));
    // the total bounds the upload; the per-sequence check then runs while the copies are in flight
    if ((uint64_t)offsets[n] > (uint64_t)n * kMaxInputLength + offsets[0]) {
        set_err("the offsets describe more residues than n_seqs sequences can hold");
        return XTN_ERR_ARG;
    }
    XTN_CK(cudaSetDevice(c->device));
    XTN_TRY(upload(c, seqs, offsets, n));
    if (check_offsets(offsets, n) != XTN_SUCCESS) {
        cudaStreamSynchronize(c->stream);  // the copies read the caller's buffers
        return XTN_ERR_ARG;
    }
    const uint8_t* dch = P<uint8_t>(c->chars);
    const uint32_t* dof = P<uint32_t>(c->offs);
    if (info && args->info_len < 1) {
        set_err("invalid info length");
        return XTN_ERR_ARG;
    }
    int r;
    begin_run(c);  // every path below reaches end_run
    if (info) {
        r = ensure(c->info, sizeof(xtn_seq_info) * (size_t)n);
        if (r == XTN_SUCCESS) {
            const cudaError_t e = cudaMemcpyAsync(c->info.p, info, sizeof(xtn_seq_info) * (size_t)n,
                                                  cudaMemcpyHostToDevice, c->stream);
            if (e != cudaSuccess) {
                set_err(std::string("copy of the sequence info failed: ") + cudaGetErrorString(e));
                r = XTN_ERR_CUDA;
            }
        }
        if (r == XTN_SUCCESS)
            r = run_overlap(c, dch, dof, P<xtn_seq_info>(c->info), n, args->distance, args->measure, args->info_len,
                            false);
    } else {
        r = run_nn(c, dch, dof, nullptr, n, args->distance, args->measure, false);
    }
    end_run(c);
    if (r != XTN_SUCCESS) return r;
    if (args->verbose) {
        const xtn_stats& st = c->stats;
        printf("xtn_b200: seqs %lld variants %lld groups %lld candidates %lld output %lld (%.3f ms device)\n",
               (long long)st.n_seqs, (long long)st.n_variants, (long long)st.n_groups, (long long)st.n_candidates,
               (long long)st.n_out, st.ms_total);
    }
    return deliver(c, cb, user);
}

int xtn_context_set_option(xtn_context* c, const char* name, int64_t v) {
    if (!c || !name) return XTN_ERR_ARG;
    if (!strcmp(name, "engine") && (v == 0 || v == 1)) c->engine = (int)v;
    else if (!strcmp(name, "bucket_bits_max") && v >= 1 && v <= 14) c->bucket_bits_max = (int)v;
    else if (!strcmp(name, "group_cap") && v >= 2 && v <= kGroupCap) c->group_cap = (uint32_t)v;
    else if (!strcmp(name, "scatter_ctas_per_sm") && v >= 0 && v <= 4) c->scatter_ctas_per_sm = (int)v;
    else if (!strcmp(name, "group_tma") && (v == 0 || v == 1)) c->group_tma = (int)v;
    else if (!strcmp(name, "onesweep") && (v == 0 || v == 1)) c->onesweep = (int)v;
    else if (!strcmp(name, "pair_dedup") && v >= 0 && v <= 2) c->pair_dedup = (int)v;
    else if (!strcmp(name, "key_tables") && (v == 0 || v == 1)) c->key_tables = (int)v;
    else if (!strcmp(name, "stage_chunk") && (v == 2048 || v == 4096 || v == 8192)) c->stage_chunk = (int)v;
    else if (!strcmp(name, "split_chunk") && (v == 0 || v == 2048 || v == 4096 || v == 8192)) c->split_chunk = (int)v;
    else if (!strcmp(name, "split_slices") && (v == 1 || v == kSplitSlices)) c->split_slices = (int)v;
    else if (!strcmp(name, "wait_polls") && v >= 1 && v <= (int64_t)kScanPollLimit) c->wait_polls = (uint32_t)v;
    else if (!strcmp(name, "memory_budget") && v >= 0) c->memory_budget = v;
    else if (!strcmp(name, "max_round_records") && v >= 0) c->max_round_records = v;
    else if (!strcmp(name, "round_overlap") && (v == 0 || v == 1)) c->round_overlap = (int)v;
    else if (!strcmp(name, "graph") && (v == 0 || v == 1)) c->graph_mode = (int)v;
    else if (!strcmp(name, "verify_per") && (v == 1 || v == 4 || v == 8)) c->verify_per = (int)v;
    else if (!strcmp(name, "autotune") && (v == 0 || v == 1)) c->autotune_auto = (int)v;
    else if (!strcmp(name, "group_persistent") && (v == 0 || v == 1)) c->group_persistent = (int)v;
    else if (!strcmp(name, "shard_count") && v >= 1 && v <= kMaxShards) c->shard_count = (int)v;
    else if (!strcmp(name, "flat_gen") && (v == 0 || v == 1)) c->flat_gen = (int)v;
    else if (!strcmp(name, "split_fill") && v >= 25 && v <= 95) c->split_fill = (int)v;
    else if (!strcmp(name, "split_slotted") && (v == 0 || v == 1)) c->split_slotted = (int)v;
    else if (!strcmp(name, "shard_index") && v >= 0 && v < kMaxShards) c->shard_index = (int)v;
    else if (!strcmp(name, "wait_fault_test") && (v == 0 || v == 1)) c->wait_fault_test = (int)v;
    else if (!strcmp(name, "dedup_slots_log2") && (v == 0 || (v >= 16 && v <= 30))) c->dedup_slots_log2 = (int)v;
    else {
        set_err(std::string("unknown option or value out of range: ") + name);
        return XTN_ERR_ARG;
    }
    return XTN_SUCCESS;
}

int xtn_context_autotune(xtn_context* c, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                         int32_t n, int32_t repeats, char* report, int32_t report_cap) {
    if (!c || !d_seqs || !d_offsets || n < 1) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    XTN_TRY(check_args(args));
    XTN_CK(cudaSetDevice(c->device));
    return autotune(c, args, reinterpret_cast<const uint8_t*>(d_seqs), d_offsets, n, repeats, report, report_cap);
}

int xtn_context_set_profiling(xtn_context* c, int on) {
    if (!c) return XTN_ERR_ARG;
    c->prof.on = on != 0;
    return XTN_SUCCESS;
}

int xtn_context_profile_only(xtn_context* c, const char* name) {
    if (!c) return XTN_ERR_ARG;
    c->prof.only = name ? name : "";
    return XTN_SUCCESS;
}

int xtn_context_kernel_times(const xtn_context* c, const char** names, double* ms, int64_t* launches, int cap) {
    if (!c) return -XTN_ERR_ARG;
    int n = (int)c->kt_names.size();
    for (int i = 0; i < n && i < cap; i++) {
        if (names) names[i] = c->kt_names[i].c_str();
        if (ms) ms[i] = c->kt_ms[i];
        if (launches) launches[i] = c->kt_launches[i];
    }
    return n;
}

int xtn_context_fetch(xtn_context* c, xtn_int2* pairs, int8_t* distances, uint64_t* freqs, int64_t cap) {
    if (!c || cap < 0) return XTN_ERR_ARG;
    int64_t m = std::min(cap, c->n_out);
    if (m <= 0) return XTN_SUCCESS;
    if (pairs) XTN_CK(cudaMemcpyAsync(pairs, c->out_pairs.p, sizeof(xtn_int2) * m, cudaMemcpyDeviceToHost, c->stream));
    if (distances && !c->overlap_result)
        XTN_CK(cudaMemcpyAsync(distances, c->out_dist.p, (size_t)m, cudaMemcpyDeviceToHost, c->stream));
    if (freqs && c->overlap_result)
        XTN_CK(cudaMemcpyAsync(freqs, c->out_freq.p, sizeof(uint64_t) * m, cudaMemcpyDeviceToHost, c->stream));
    XTN_CK(cudaStreamSynchronize(c->stream));
    return XTN_SUCCESS;
}

int xtn_context_result_device(xtn_context* c, const xtn_int2** d_pairs, const int8_t** d_dist, int64_t* n_out) {
    if (!c) return XTN_ERR_ARG;
    if (d_pairs) *d_pairs = P<xtn_int2>(c->out_pairs);
    if (d_dist) *d_dist = P<int8_t>(c->out_dist);
    if (n_out) *n_out = c->n_out;
    return XTN_SUCCESS;
}

}  // extern "C"

// ------------------------------------------------------------------ shard exchange
// A sharded search (options shard_count / shard_index) leaves on each rank the verified pairs
// of its first-level buckets, sorted by (x, y); a pair whose sequences share variants in the
// buckets of several shards is found by each of them. The exchange gives every rank the pairs
// whose x lies in its id range, [ceil(k n / K), ceil((k + 1) n / K)) for rank k of K, as one
// 64-bit key per pair, x << (b + 8) | y << 8 | distance with b = id bits of n: the sorted
// output splits into contiguous runs per owner, and the owner's merge (sort, unique) restores
// the reference's sorted, duplicate-free order over its range, so that the ranks' outputs in
// rank order are the whole search's output.
namespace xtn {

__global__ void k_result_keys(const xtn_int2* __restrict__ pairs, const int8_t* __restrict__ dist, int64_t m, int b,
                              uint64_t* __restrict__ keys) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const xtn_int2 p = pairs[i];
    keys[i] = ((uint64_t)(uint32_t)p.x << (b + 8)) | ((uint64_t)(uint32_t)p.y << 8) | (uint64_t)(uint8_t)dist[i];
}

// starts[k] = first index of the sorted pairs whose x >= ceil(k n / K) (starts[K] = m).
__global__ void k_range_starts(const xtn_int2* __restrict__ pairs, int64_t m, int64_t n, int K,
                               int64_t* __restrict__ starts) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > K) return;
    if (k == K) {
        starts[k] = m;
        return;
    }
    const int64_t x0 = ((int64_t)k * n + K - 1) / K;
    int64_t lo = 0, hi = m;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)pairs[mid].x < x0) lo = mid + 1;
        else hi = mid;
    }
    starts[k] = lo;
}

__global__ void k_key_heads(const uint64_t* __restrict__ keys, int64_t m, uint8_t* __restrict__ head) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

__global__ void k_key_compact(const uint64_t* __restrict__ keys, int64_t m, int b, const uint8_t* __restrict__ head,
                              const uint32_t* __restrict__ pos, xtn_int2* __restrict__ out, int8_t* __restrict__ dist) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || !head[i]) return;
    const uint64_t k = keys[i];
    const uint32_t o = pos[i];
    const uint64_t idmask = (1ull << b) - 1ull;
    out[o] = xtn_int2{(int32_t)(k >> (b + 8)), (int32_t)((k >> 8) & idmask)};
    dist[o] = (int8_t)(uint8_t)(k & 0xffu);
}

static int key_bits_for(xtn_context* c, int32_t n_seqs, int* b) {
    *b = id_bits_for(n_seqs);
    if (2 * *b + 8 > 64) {
        set_err("too many sequences for 64-bit pair keys");
        return XTN_ERR_LIMIT;
    }
    return XTN_SUCCESS;
}

}  // namespace xtn

extern "C" {

int xtn_context_result_keys(xtn_context* c, int32_t n_seqs, uint64_t* d_keys, int64_t capacity, int32_t n_ranges,
                            int64_t* range_starts) {
    if (!c || n_seqs < 1 || n_ranges < 1 || n_ranges > kMaxShards || !range_starts || (c->n_out > 0 && !d_keys)) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    if (c->overlap_result) {
        set_err("the last result is an overlap matrix, not pairs");
        return XTN_ERR_ARG;
    }
    if (capacity < c->n_out) {
        set_err("the key buffer holds fewer entries than the result");
        return XTN_ERR_ARG;
    }
    int b = 0;
    XTN_TRY(key_bits_for(c, n_seqs, &b));
    XTN_CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const int64_t m = c->n_out;
    if (m > 0)
        XTN_LAUNCH("result_keys", k_result_keys<<<blocks_for(m), kThreads, 0, s>>>(
                                      P<xtn_int2>(c->out_pairs), P<int8_t>(c->out_dist), m, b, d_keys));
    XTN_TRY(ensure(c->scratch64, sizeof(int64_t) * (n_ranges + 1)));
    XTN_LAUNCH("range_starts", k_range_starts<<<blocks_for(n_ranges + 1), kThreads, 0, s>>>(
                                   P<xtn_int2>(c->out_pairs), m, n_seqs, n_ranges, P<int64_t>(c->scratch64)));
    XTN_CK(cudaGetLastError());
    XTN_CK(cudaMemcpyAsync(range_starts, c->scratch64.p, sizeof(int64_t) * (n_ranges + 1), cudaMemcpyDeviceToHost, s));
    XTN_CK(cudaStreamSynchronize(s));
    return XTN_SUCCESS;
}

int xtn_context_merge_keys(xtn_context* c, int32_t n_seqs, const uint64_t* d_keys, int64_t count, int64_t* n_out) {
    if (!c || n_seqs < 1 || count < 0 || (count > 0 && !d_keys) || count >= (int64_t)UINT32_MAX) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    int b = 0;
    XTN_TRY(key_bits_for(c, n_seqs, &b));
    XTN_CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    memset(&c->stats, 0, sizeof c->stats);
    c->overlap_result = false;
    c->n_out = 0;
    if (count > 0) {
        XTN_TRY(ensure(c->pairA, sizeof(uint64_t) * count + 64));
        XTN_TRY(ensure(c->pairB, sizeof(uint64_t) * count + 64));
        XTN_CK(cudaMemcpyAsync(c->pairB.p, d_keys, sizeof(uint64_t) * count, cudaMemcpyDeviceToDevice, s));
        uint64_t* keys = P<uint64_t>(c->pairB);
        if (count > 1)
            XTN_TRY(sort_u64(c, c->pairB, c->pairA, count, 0, 2 * b + 8, &keys, XTN_SORT_NAMES("shard_key_sort")));
        XTN_TRY(ensure(c->flag, (size_t)count));
        XTN_TRY(ensure(c->fpos, sizeof(uint32_t) * (count + 1)));
        XTN_LAUNCH("key_heads", k_key_heads<<<blocks_for(count), kThreads, 0, s>>>(keys, count, P<uint8_t>(c->flag)));
        XTN_TRY((scan_1p<uint8_t, uint32_t>(c, P<uint8_t>(c->flag), P<uint32_t>(c->fpos), count)));
        XTN_TRY(ensure(c->out_pairs, sizeof(xtn_int2) * count));
        XTN_TRY(ensure(c->out_dist, (size_t)count));
        XTN_LAUNCH("key_compact", k_key_compact<<<blocks_for(count), kThreads, 0, s>>>(
                                      keys, count, b, P<uint8_t>(c->flag), P<uint32_t>(c->fpos),
                                      P<xtn_int2>(c->out_pairs), P<int8_t>(c->out_dist)));
        XTN_CK(cudaGetLastError());
        uint64_t u = 0;
        XTN_TRY(read_scalar(c, P<uint32_t>(c->fpos) + count, 4, &u));
        c->n_out = (int64_t)u;
    }
    c->stats.n_out = c->n_out;
    c->stats.n_seqs = n_seqs;
    if (n_out) *n_out = c->n_out;
    return XTN_SUCCESS;
}

// ------------------------------------------------------------------ sharded search with exchange
// One search over K ranks, each holding the whole input (for verification) and generating the
// variants of its own sequences [rank n / K, (rank + 1) n / K) only. xtn_shard_generate:
// length check, pack and variant offsets of all sequences (the first-level shape depends on
// the whole search, so every rank derives the same one), then the two-pass first level over the
// rank's own sequences: their records, partitioned into the search's first-level buckets, in
// the context's record buffer A, and the per-bucket counts on the host. The ranks then sum the
// counts, give each rank a contiguous range of buckets, and send each owner its buckets'
// records (xtn.nn_sharded_exchange: two all-to-alls). xtn_shard_search gathers what a rank
// received into contiguous buckets and runs the rest of the search on them (plan, split,
// grouping, pair dedup, sort, verification); the exchange of verified pairs by owner follows.
extern "C" int xtn_shard_generate(xtn_context* c, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                                  int32_t n, int32_t rank, int32_t n_ranks, uint64_t* bucket_counts, int32_t cap,
                                  int32_t* n_buckets, const uint64_t** d_records, int64_t* n_records) {
    if (!c || !d_seqs || !d_offsets || n < 1 || n_ranks < 1 || n_ranks > kMaxShards || rank < 0 || rank >= n_ranks ||
        !n_buckets || !d_records || !n_records || (cap > 0 && !bucket_counts)) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    XTN_TRY(check_args(args));
    const int d = args->distance;
    if (d > 2 || !c->key_tables || c->stage_chunk != 4096) {
        set_err("the sharded exchange needs distance <= 2, the key tables and stage_chunk 4096");
        return XTN_ERR_ARG;
    }
    XTN_CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    begin_run(c);
    const uint8_t* chars = reinterpret_cast<const uint8_t*>(d_seqs);
    xtn_stats& st = c->stats;
    memset(&st, 0, sizeof st);
    st.n_seqs = n;
    st.id_bits = id_bits_for(n);
    uint64_t V = 0;
    int r = pack_and_count(c, chars, d_offsets, nullptr, n, d, true, &V);
    if (r != XTN_SUCCESS) {
        end_run(c);
        return r;
    }
    st.n_variants = (int64_t)V;
    BucketPlan bp;
    bucket_shape(c, n, d, V, &bp, true);
    const int nb = bp.nb, b1 = bp.b1;
    // this rank's sequences and their tiles (the partition and the histograms use the same)
    const int s0 = (int)((int64_t)n * rank / n_ranks), s1 = (int)((int64_t)n * (rank + 1) / n_ranks);
    const int nr = s1 - s0;
    const int64_t wave = (int64_t)c->sms * ctas_per_sm_for<ScatterSmem<StageLarge>>();
    const int ntiles = nr > 0 ? (int)(wave * std::max<int64_t>(1, ((int64_t)nr + wave * 4096 - 1) / (wave * 4096))) : 0;
    const int tile = ntiles > 0 ? (nr + ntiles - 1) / ntiles : 1;
    uint64_t rec0 = 0, rec1 = 0;
    r = read_scalar(c, P<uint64_t>(c->voff) + s0, 8, &rec0);
    if (r == XTN_SUCCESS) r = read_scalar(c, P<uint64_t>(c->voff) + s1, 8, &rec1);
    const uint64_t Vr = rec1 - rec0;
    if (r == XTN_SUCCESS && Vr >= (uint64_t)UINT32_MAX - (uint64_t(1) << 20)) {
        set_err("too many records for one rank (" + std::to_string(Vr) + "): use more ranks");
        r = XTN_ERR_LIMIT;
    }
    auto run = [&]() -> int {
        XTN_TRY(bucket_reserve(c, bp, n, d, V));
        XTN_TRY(ensure(c->bcounts, sizeof(uint32_t) * (size_t)std::max(1, ntiles) * nb));
        XTN_TRY(ensure(c->boffs, sizeof(uint32_t) * (size_t)std::max(1, ntiles) * nb));
        XTN_TRY(bucket_attrs(c));
        if (d >= 2) XTN_TRY(build_task_map(c, n, &bp));
        XTN_TRY(ensure(c->recA, sizeof(uint64_t) * Vr + 64));
        XTN_TRY(ensure(c->recB, sizeof(uint64_t) * Vr + 64));
        XTN_TRY(ensure(c->bcnt, 64));
        XTN_CK(cudaMemsetAsync(c->bcnt.p, 0, 64, s));
        if (ntiles > 0) {
            XTN_LAUNCH("bucket_gen", (k_bucket_gen<kBucketThreads, 2><<<ntiles, kBucketThreads, sizeof(uint32_t) * nb, s>>>(
                                         P<uint8_t>(c->klen), P<uint64_t>(c->runinfo), P<uint64_t>(c->ktab),
                                         P<uint64_t>(c->voff), P<uint64_t>(c->toff), bp.tseq, s1, tile, d, b1,
                                         id_bits_for(n), P<uint64_t>(c->recB), P<uint32_t>(c->bcounts), nullptr, s0,
                                         rec0)));
            XTN_LAUNCH("bucket_colscan", k_bucket_colscan<<<(nb + 31) / 32, kColscanWarps * 32, 0, s>>>(
                                             P<uint32_t>(c->bcounts), ntiles, nb, P<uint32_t>(c->boffs),
                                             P<uint32_t>(c->btotals)));
            XTN_TRY(scan_u32_to_u64(c, P<uint32_t>(c->btotals), P<uint64_t>(c->bstart), nb));
            XTN_LAUNCH("bucket_partition",
                       k_bucket_partition<StageHuge><<<ntiles, StageHuge::kThreads, sizeof(StageSmem<StageHuge>), s>>>(
                           P<uint64_t>(c->recB), P<uint64_t>(c->voff), s1, tile, b1, id_bits_for(n),
                           P<uint32_t>(c->boffs), P<uint64_t>(c->bstart), P<uint64_t>(c->recA),
                           P<unsigned int>(c->bcnt), nullptr, s0, rec0));
        } else {
            XTN_CK(cudaMemsetAsync(c->btotals.p, 0, sizeof(uint32_t) * nb, s));
        }
        XTN_CK(cudaGetLastError());
        std::vector<uint32_t> tot(nb);
        XTN_CK(cudaMemcpyAsync(tot.data(), c->btotals.p, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost, s));
        XTN_CK(cudaMemcpyAsync(c->h_scalar, c->bcnt.p, 32, cudaMemcpyDeviceToHost, s));
        XTN_CK(cudaStreamSynchronize(s));
        uint32_t cnt[8];
        memcpy(cnt, c->h_scalar, 32);
        if (cnt[kCntWaitFail] != 0) {
            set_err("bucket partition: " + std::to_string(cnt[kCntWaitFail]) + " chunk copies did not complete in time");
            return XTN_ERR_CUDA;
        }
        for (int k = 0; k < nb && k < cap; k++) bucket_counts[k] = tot[k];
        return XTN_SUCCESS;
    };
    if (r == XTN_SUCCESS) r = run();
    end_run(c);
    if (r != XTN_SUCCESS) return r;
    *n_buckets = nb;
    *d_records = P<uint64_t>(c->recA);
    *n_records = (int64_t)Vr;
    return XTN_SUCCESS;
}

extern "C" int xtn_shard_search(xtn_context* c, const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets,
                                int32_t n, const uint64_t* d_records, const uint64_t* piece_counts, int32_t n_pieces,
                                int32_t b_n, int64_t* n_out) {
    if (!c || !d_seqs || !d_offsets || n < 1 || n_pieces < 1 || b_n < 0 || (b_n > 0 && !piece_counts)) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    XTN_TRY(check_args(args));
    XTN_CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const uint8_t* chars = reinterpret_cast<const uint8_t*>(d_seqs);
    const int d = args->distance, idbits = id_bits_for(n);
    // the buckets' totals and starts, and one gather run per (bucket, piece)
    std::vector<uint64_t> bstart((size_t)b_n + 1, 0), piece_base((size_t)n_pieces + 1, 0);
    for (int p = 0; p < n_pieces; p++) {
        uint64_t t = 0;
        for (int k = 0; k < b_n; k++) t += piece_counts[(size_t)p * b_n + k];
        piece_base[p + 1] = piece_base[p] + t;
    }
    for (int k = 0; k < b_n; k++) {
        uint64_t t = 0;
        for (int p = 0; p < n_pieces; p++) t += piece_counts[(size_t)p * b_n + k];
        bstart[k + 1] = bstart[k] + t;
    }
    const uint64_t V = bstart[b_n];
    if (V > 0 && !d_records) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    if (V >= (uint64_t)UINT32_MAX - (uint64_t(1) << 20)) {
        set_err("too many records for one rank's buckets (" + std::to_string(V) + ")");
        return XTN_ERR_LIMIT;
    }
    std::vector<GatherRun> runs;
    {
        std::vector<uint64_t> in_piece(n_pieces, 0);
        for (int k = 0; k < b_n; k++) {
            uint64_t dst = bstart[k];
            for (int p = 0; p < n_pieces; p++) {
                const uint64_t m = piece_counts[(size_t)p * b_n + k];
                if (m) runs.push_back(GatherRun{piece_base[p] + in_piece[p], dst, m});
                in_piece[p] += m;
                dst += m;
            }
        }
    }
    begin_run(c);
    xtn_stats& st = c->stats;
    memset(&st, 0, sizeof st);
    st.n_seqs = n;
    st.n_rounds = 1;
    st.id_bits = idbits;
    st.n_variants = (int64_t)V;
    auto run = [&]() -> int {
        XTN_CK(cudaEventRecord(c->ev[0], s));
        XTN_TRY(ensure(c->recA, sizeof(uint64_t) * V + 64));
        XTN_TRY(ensure(c->bstart, sizeof(uint64_t) * (b_n + 1)));
        XTN_TRY(ensure(c->gruns, sizeof(GatherRun) * std::max<size_t>(1, runs.size())));
        XTN_CK(cudaMemcpyAsync(c->bstart.p, bstart.data(), sizeof(uint64_t) * (b_n + 1), cudaMemcpyHostToDevice, s));
        if (!runs.empty()) {
            XTN_CK(cudaMemcpyAsync(c->gruns.p, runs.data(), sizeof(GatherRun) * runs.size(), cudaMemcpyHostToDevice, s));
            XTN_LAUNCH("gather_runs", k_gather_runs<<<(unsigned)runs.size(), 256, 0, s>>>(P<GatherRun>(c->gruns), d_records,
                                                                                         P<uint64_t>(c->recA)));
        }
        XTN_CK(cudaEventRecord(c->ev[1], s));
        XTN_TRY(bucket_attrs(c));
        BucketPlan bp;
        bp.nb = b_n;
        bp.slotted = c->split_slotted != 0;
        uint64_t Pc = 0;
        XTN_TRY(ensure(c->counter, 64));
        if (b_n > 0) {
            XTN_TRY(bucket_round(c, bp, n, d, idbits, 0, (uint32_t)b_n, 0, V, c->pairA, 0, &Pc, true));
        } else {  // a rank that owns no bucket: the bucket stages take no time
            for (int k = 2; k <= 4; k++) XTN_CK(cudaEventRecord(c->ev[k], s));
        }
        c->last_pc_per_rec = V ? (double)Pc / (double)V : 0.0;
        st.n_candidates = (int64_t)Pc;
        return nn_tail(c, chars, d_offsets, nullptr, n, d, args->measure, Pc, false);
    };
    const int r = run();
    end_run(c);
    if (r == XTN_SUCCESS && n_out) *n_out = c->n_out;
    return r;
}

static std::mutex g_default_mu;
static xtn_context* g_default = nullptr;

int xtn_perform(const xtn_args* args, const char* seqs, const uint32_t* offsets, int32_t n, const xtn_seq_info* info,
                xtn_callback cb, void* user) {
    std::lock_guard<std::mutex> lk(g_default_mu);
    if (!g_default) XTN_TRY(xtn_context_create(0, &g_default));
    return xtn_context_perform(g_default, args, seqs, offsets, n, info, cb, user);
}

}  // extern "C"

#include "xtn_index.cuh"

// ------------------------------------------------------------------ search without allocation
// Some callers cannot allocate device memory while they run: a host whose framework caching
// allocator already owns the device's memory (so a raw cudaMalloc can fail or fragment it),
// a latency-critical loop that must not pay the device-wide synchronisation cudaMalloc and
// cudaFree can cause, or a plugin host whose policy forbids allocation on the call path. For
// them, xtn_nn_search_static runs the nearest-neighbour search (the sort-engine kernels)
// with all of its scratch carved out of one file-scope device array of fixed size. The caller
// passes the inputs and the output buffers; the entry point calls no cudaMalloc, cudaFree or
// allocating library routine.
namespace xtn {

constexpr size_t kStaticArenaBytes = size_t(32) << 20;  // 32 MiB, held by every GPU that loads the library
constexpr int kStaticMaxSeqs = 4096;
constexpr int kStaticMaxDevices = 64;

__device__ __align__(256) unsigned char g_static_arena[kStaticArenaBytes];

// Device address of g_static_arena per device (the host-side name is only a stand-in),
// resolved once per device with that device current.
static std::mutex g_static_mu;
static void* g_static_addr[kStaticMaxDevices] = {};

static int static_arena(int device, unsigned char** out) {
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_arena);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_err(std::string("cudaGetSymbolAddress of the static scratch array failed: ") + cudaGetErrorString(e));
            return XTN_ERR_CUDA;
        }
        g_static_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_static_addr[device]);
    return XTN_SUCCESS;
}

// Bump allocator over the arena.
struct Carver {
    unsigned char* base;
    size_t used, cap;
    template <typename T>
    bool take(T** p, size_t count) {
        size_t bytes = (sizeof(T) * count + 64 + 255) & ~size_t(255);
        if (used + bytes > cap) return false;
        *p = reinterpret_cast<T*>(base + used);
        used += bytes;
        return true;
    }
};

static int arena_full(const char* what) {
    set_err(std::string("input exceeds the static scratch array (") + std::to_string(kStaticArenaBytes >> 20) +
            " MiB) at: " + what);
    return XTN_ERR_LIMIT;
}

static int read_u64(const void* d, size_t bytes, cudaStream_t s, uint64_t* out) {
    uint64_t v = 0;
    XTN_CK(cudaMemcpyAsync(&v, d, bytes, cudaMemcpyDeviceToHost, s));
    XTN_CK(cudaStreamSynchronize(s));
    *out = v;
    return XTN_SUCCESS;
}

static int nn_search_static(const uint8_t* chars, const uint32_t* offs, int n, int d, int measure, xtn_int2* out_pairs,
                            int8_t* out_dist, int64_t out_cap, int64_t* n_out, cudaStream_t s, unsigned char* arena) {
    Carver cv{arena, 0, kStaticArenaBytes};
    const int idbits = id_bits_for(n);
    u128* keys;
    uint8_t* klen;
    uint32_t* vcnt;
    uint64_t *voff, *runinfo, *scan64;
    unsigned long long* counter;
    unsigned int* lenbad;
    if (!cv.take(&keys, n) || !cv.take(&klen, n) || !cv.take(&vcnt, n) || !cv.take(&voff, n + 1) ||
        !cv.take(&runinfo, n) || !cv.take(&scan64, scan_scratch_elems(n)) || !cv.take(&counter, 2) ||
        !cv.take(&lenbad, 1))
        return arena_full("sequence tables");
    // the caller's offsets are checked on the device (1..500 residues each) before any kernel
    // that indexes by length runs
    XTN_CK(cudaMemsetAsync(lenbad, 0xff, 4, s));
    XTN_LAUNCH("check_lengths", k_check_lengths<<<blocks_for(n), kThreads, 0, s>>>(offs, nullptr, n, lenbad));
    XTN_LAUNCH("pack", k_pack<<<blocks_for(n, kPackThreads), kPackThreads, 0, s>>>(chars, offs, nullptr, n, d, keys, klen, vcnt, runinfo,
                                                                 nullptr));
    XTN_CK(cudaGetLastError());
    scan_exclusive<uint32_t, uint64_t>(vcnt, voff, n, scan64, s);
    uint64_t V = 0, bad = 0;
    XTN_TRY(read_u64(lenbad, 4, s, &bad));
    if ((uint32_t)bad != 0xffffffffu) {
        set_err("sequence " + std::to_string((uint32_t)bad) + " has an invalid length");
        return XTN_ERR_ARG;
    }
    XTN_TRY(read_u64(voff + n, 8, s, &V));
    uint64_t *recA, *recB;
    uint32_t* rscratch;
    if (!cv.take(&recA, V) || !cv.take(&recB, V) || !cv.take(&rscratch, radix_scratch_elems((int64_t)V)))
        return arena_full("variant records");
    XTN_LAUNCH("gen", k_gen<<<blocks_for(n), kThreads, 0, s>>>(keys, klen, runinfo, nullptr, voff, n, d, idbits, recA));
    uint64_t* recs = radix_sort_u64(recA, recB, (int64_t)V, idbits, 64, rscratch, s, "key_sort_upsweep",
                                    "key_sort_downsweep");
    // groups: at most one per two records
    const int64_t gcap = (int64_t)(V / 2 + 1);
    uint64_t *gstart, *gcnt, *goff;
    uint32_t* gsize;
    if (!cv.take(&gstart, gcap) || !cv.take(&gsize, gcap) || !cv.take(&gcnt, gcap + 1) || !cv.take(&goff, gcap + 1))
        return arena_full("groups");
    XTN_CK(cudaMemsetAsync(counter, 0, 16, s));
    XTN_LAUNCH("find_groups", k_find_groups<<<blocks_for((int64_t)V), kThreads, 0, s>>>(recs, (int64_t)V, idbits,
                                                                                         gstart, gsize, counter, gcap));
    XTN_CK(cudaGetLastError());
    uint64_t G = 0, Pc = 0;
    XTN_TRY(read_u64(counter, 8, s, &G));
    uint64_t* scanG;
    if (!cv.take(&scanG, scan_scratch_elems((int64_t)G + 1))) return arena_full("group scan");
    if (G > 0) {
        XTN_LAUNCH("pair_counts", k_pair_counts<<<blocks_for((int64_t)G), kThreads, 0, s>>>(gsize, (int64_t)G, gcnt));
        scan_exclusive<uint64_t, uint64_t>(gcnt, goff, (int64_t)G, scanG, s);
        XTN_TRY(read_u64(goff + G, 8, s, &Pc));
    }
    uint64_t *pairA, *pairB;
    uint32_t *pscratch, *fpos;
    int8_t* dist;
    uint8_t* flag;
    if (Pc >= (uint64_t)UINT32_MAX || !cv.take(&pairA, Pc) || !cv.take(&pairB, Pc) || !cv.take(&dist, Pc) ||
        !cv.take(&flag, Pc) || !cv.take(&fpos, Pc + 1) ||
        !cv.take(&pscratch, std::max<int64_t>(radix_scratch_elems((int64_t)Pc), scan_scratch_elems((int64_t)Pc))))
        return arena_full("candidate pairs");
    uint64_t nout = 0;
    if (Pc > 0) {
        uint64_t threads = (Pc + kEmitPer - 1) / kEmitPer;
        XTN_LAUNCH("emit", k_emit<<<blocks_for((int64_t)threads), kThreads, 0, s>>>(recs, gstart, gsize, goff,
                                                                                      (int64_t)G, Pc, idbits, pairA));
        uint64_t* pairs = Pc > 1 ? radix_sort_u64(pairA, pairB, (int64_t)Pc, 0, 2 * idbits, pscratch, s,
                                                  "pair_sort_upsweep", "pair_sort_downsweep")
                                 : pairA;
        launch_verify(kVerifyPer, pairs, (int64_t)Pc, idbits, chars, offs, nullptr, d, measure, dist, flag, nullptr, s);
        scan_exclusive<uint8_t, uint32_t>(flag, fpos, (int64_t)Pc, pscratch, s);
        XTN_TRY(read_u64(fpos + Pc, 4, s, &nout));
        if ((int64_t)nout > out_cap) {
            *n_out = (int64_t)nout;
            set_err("output buffer too small: " + std::to_string(nout) + " pairs");
            return XTN_ERR_LIMIT;
        }
        if (nout > 0)
            XTN_LAUNCH("compact", k_compact<<<blocks_for((int64_t)Pc), kThreads, 0, s>>>(pairs, (int64_t)Pc, idbits,
                                                                                          dist, flag, fpos, out_pairs,
                                                                                          out_dist, nullptr));
    }
    XTN_CK(cudaGetLastError());
    XTN_CK(cudaStreamSynchronize(s));
    *n_out = (int64_t)nout;
    return XTN_SUCCESS;
}

}  // namespace xtn

extern "C" int xtn_nn_search_static(const xtn_args* args, const char* d_seqs, const uint32_t* d_offsets, int32_t n_seqs,
                                    xtn_int2* d_out_pairs, int8_t* d_out_distances, int64_t out_cap, int64_t* n_out,
                                    void* stream) {
    if (!d_seqs || !d_offsets || !n_out || n_seqs < 1 || out_cap < 0 || (out_cap > 0 && (!d_out_pairs || !d_out_distances))) {
        set_err("invalid arguments");
        return XTN_ERR_ARG;
    }
    XTN_TRY(check_args(args));
    if (n_seqs > kStaticMaxSeqs) {
        set_err("xtn_nn_search_static accepts at most " + std::to_string(kStaticMaxSeqs) + " sequences (got " +
                std::to_string(n_seqs) + ")");
        return XTN_ERR_LIMIT;
    }
    int device = 0;
    XTN_CK(cudaGetDevice(&device));
    if (device < 0 || device >= kStaticMaxDevices) {
        set_err("device index beyond the static scratch table");
        return XTN_ERR_LIMIT;
    }
    unsigned char* arena = nullptr;
    XTN_TRY(static_arena(device, &arena));
    return nn_search_static(reinterpret_cast<const uint8_t*>(d_seqs), d_offsets, n_seqs, args->distance, args->measure,
                            d_out_pairs, d_out_distances, out_cap, n_out, static_cast<cudaStream_t>(stream), arena);
}
