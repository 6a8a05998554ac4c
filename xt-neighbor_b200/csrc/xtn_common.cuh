// Host+device helpers shared by the sm_100a kernels and the CPU self-test.
//
// Key format. The reference keys a sequence by its first 18 residues, 5 bits each
// (S/src/codec.cu:43-60, S/src/kernel.cu:594-610, MAX_COMPRESSED_LENGTH S/src/xtn.h:8).
// Here the same 90 bits live in one unsigned 128-bit word, residue i in bits
// [123-5i, 128-5i) (MSB first) and zeros after the last residue, so a deletion is one
// masked shift and equal strings are equal words.
//
// Variant enumeration. The reference emits every deletion set of at most min(d, L)
// positions, duplicates included (S/src/generate_combination.cu:42-141). Deleting any c
// residues of one run of equal residues gives the same string as deleting the first c of
// that run, so enumerating only "run-prefix" deletion sets yields the same set of distinct
// strings with far fewer repeats. The set of key-sharing sequence pairs is unchanged; only
// repeated emissions of the same pair disappear.
#pragma once
#include <cstdint>
#include <thread>

#ifdef __CUDACC__
#define XTN_HD __host__ __device__ __forceinline__
#else
#define XTN_HD inline
#endif

namespace xtn {

typedef unsigned __int128 u128;

constexpr int kKeyLen = 18;          // S/src/xtn.h:8
constexpr int kLevenshtein = 0;      // S/src/xtn.h:12
constexpr int kHamming = 1;          // S/src/xtn.h:14
constexpr int kHammingLenMismatch = 77;  // S/src/kernel.cu:292-293
constexpr int kMaxInputLength = 500;     // S/src/codec.cu:18

// 'A'..'Y' -> 1..25 (S/src/codec.cu:25-38); inputs are validated by the parser.
XTN_HD int code_of(uint8_t c) { return (int)c - ('A' - 1); }

XTN_HD u128 key_put(u128 v, int i, unsigned code) { return v | ((u128)code << (123 - 5 * i)); }
XTN_HD int key_get(u128 v, int i) { return (int)((v >> (123 - 5 * i)) & 31u); }

// Delete residue p of a packed key (p < 18).
XTN_HD u128 key_del(u128 v, int p) {
    if (p == 0) return v << 5;
    u128 hi = ~(u128)0 << (128 - 5 * p);
    return (v & hi) | ((v << 5) & ~hi);
}

// Bit i set when residue i starts a run of equal residues (i < L).
XTN_HD uint32_t key_run_starts(u128 v, int L) {
    u128 x = v ^ (v >> 5);
    uint32_t m = 0;
    for (int i = 0; i < L; i++)
        if (key_get(x, i)) m |= 1u << i;
    return m;
}

// Variant hash. A variant string v_0..v_{m-1} (residue codes) hashes to
// hash_fin(P(v)), P(v) = sum_k v_k r^k (mod 2^64) for a fixed odd r. Only equality of
// variants matters for correctness: equal strings always get equal hashes, and pairs that
// share only a hash are removed by exact verification. The polynomial form makes every
// one- and two-deletion variant of a key a sum of two entries of a per-key table
// (key_table), so the d <= 2 paths hash a variant with one load and one add.
constexpr uint64_t kPolyR = 0x2545F4914F6CDD1DULL;

// Inverse of an odd number modulo 2^64 (Newton's iteration; each step doubles the
// correct low bits, starting from 3).
XTN_HD constexpr uint64_t inverse_odd(uint64_t a) {
    uint64_t x = a;
    for (int i = 0; i < 6; i++) x *= 2 - a * x;
    return x;
}
constexpr uint64_t kPolyRI = inverse_odd(kPolyR);
constexpr uint64_t kPolyRI2 = kPolyRI * kPolyRI;

// Xorshift-multiply finaliser: a bijection that spreads all input bits into the top bits
// (the bucket index) and the middle bits (the stored record hash).
XTN_HD uint64_t hash_fin(uint64_t x) {
    x ^= x >> 31;
    x *= 0x9E3779B97F4A7C15ULL;
    x ^= x >> 29;
    return x;
}

// The 90 key bits as two 64-bit words: residues 0..11 in a (residue i at bits [55-5i, 60-5i)),
// residues 12..17 in b (residue 12+j at bits [25-5j, 30-5j)). The hash code reads codes from
// these words with 64-bit shifts only: a Horner loop over 128-bit shifts of the key gave
// wrong values in one device kernel build (the same source, with 64-bit words, is correct).
struct KeyWords {
    uint64_t a, b;
};
XTN_HD KeyWords key_words(u128 v) { return KeyWords{(uint64_t)(v >> 68), (uint64_t)(v >> 38) & ((1ull << 30) - 1ull)}; }
XTN_HD uint32_t word_code(KeyWords w, int i) {
    return (uint32_t)(i < 12 ? (w.a >> (55 - 5 * i)) & 31u : (w.b >> (25 - 5 * (i - 12))) & 31u);
}

// P of a packed key, by Horner's rule from the last position (zero padding adds nothing).
XTN_HD uint64_t key_poly(u128 v) {
    const KeyWords w = key_words(v);
    uint64_t acc = 0;
    for (int i = kKeyLen - 1; i >= 0; i--) acc = acc * kPolyR + word_code(w, i);
    return acc;
}

XTN_HD uint64_t key_hash(u128 v) { return hash_fin(key_poly(v)); }

// Per-key hash table. With prefix sums P_i = sum_{j<i} c_j r^j of the key's codes and
// P_L its full polynomial, deleting p < q gives
//   P(del p,q) = P_p + r^-1 (P_q - P_{p+1}) + r^-2 (P_L - P_{q+1}) = K[p] + G[q]
//   G[q] = r^-1 P_q - r^-2 P_{q+1},   K[p] = P_p - r^-1 P_{p+1} + r^-2 P_L = r G[p] + r^-2 P_L,
// and deleting p alone gives P_p + r^-1 (P_L - P_{p+1}) = r G[p] + r^-1 P_L. The table holds
// G[0..17] and P_L; K[p] costs one multiply-add.
constexpr int kTabG = 0;                  // G[0..17]
constexpr int kTabKey = kKeyLen;          // P_L, the key's own polynomial
constexpr int kTabLen = kKeyLen + 1;      // 19 words per key

// st(slot, value) for every slot 0..kTabLen-1 (entries past the key's length are unused).
template <class Store>
XTN_HD void key_table(u128 key, Store&& st) {
    const KeyWords w = key_words(key);
    uint64_t P = 0, pw = 1;
    for (int i = 0; i < kKeyLen; i++) {
        const uint64_t Pn = P + word_code(w, i) * pw;
        st(kTabG + i, kPolyRI * P - kPolyRI2 * Pn);
        P = Pn;
        pw *= kPolyR;
    }
    st(kTabKey, P);
}

// Calls f(key) once per run-prefix deletion set of at most min(d, L) positions
// (the empty set included). Returns the number of calls.
template <class F>
XTN_HD int for_each_variant(u128 key, int L, int d, F&& f) {
    f(key);
    int e = d < L ? d : L;
    if (e <= 0) return 1;
    uint32_t rs = key_run_starts(key, L);
    int count = 1;
    if (e <= 2) {
        for (int p = 0; p < L; p++) {
            if (!((rs >> p) & 1u)) continue;
            u128 v1 = key_del(key, p);
            f(v1);
            count++;
            if (e == 2)
                for (int q = p + 1; q < L; q++) {
                    if (!(((rs >> q) & 1u) || q == p + 1)) continue;
                    f(key_del(v1, q - 1));
                    count++;
                }
        }
        return count;
    }
    // general depth: iterative DFS over ascending run-prefix deletion sets
    int pos[kKeyLen];
    u128 val[kKeyLen + 1];
    val[0] = key;
    int depth = 0, q = 0;
    while (true) {
        if (depth < e && q < L) {
            bool ok = ((rs >> q) & 1u) || (depth > 0 && pos[depth - 1] == q - 1);
            if (ok) {
                pos[depth] = q;
                val[depth + 1] = key_del(val[depth], q - depth);
                f(val[depth + 1]);
                count++;
                depth++;
                q = q + 1;
            } else {
                q++;
            }
            continue;
        }
        if (depth == 0) break;
        depth--;
        q = pos[depth] + 1;
    }
    return count;
}

struct CountOnly {
    XTN_HD void operator()(u128) const {}
};

XTN_HD int popc32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __popc(x);
#else
    return __builtin_popcount(x);
#endif
}

// Position of the lowest set bit (x != 0).
XTN_HD int ctz32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __ffs(x) - 1;
#else
    return __builtin_ctz(x);
#endif
}

// Number of calls for_each_variant makes, in closed form for d <= 2.
XTN_HD int variant_count(u128 key, int L, int d) {
    int e = d < L ? d : L;
    if (e <= 0) return 1;
    if (e <= 2) {
        uint32_t rs = key_run_starts(key, L);
        int R = popc32(rs);
        if (e == 1) return 1 + R;
        uint32_t cont = ~rs & ((L >= 32) ? 0xffffffffu : ((1u << L) - 1u));
        int R2 = popc32(rs & (cont >> 1));
        return 1 + R + R * (R - 1) / 2 + R2;
    }
    return for_each_variant(key, L, d, CountOnly{});
}

// Position of the k-th (0-based) set bit of m (m has more than k set bits).
XTN_HD int select_bit(uint32_t m, int k) {
    int p = 0, c;
    c = popc32(m & 0xffffu);
    if (k >= c) { k -= c; m >>= 16; p += 16; }
    c = popc32(m & 0xffu);
    if (k >= c) { k -= c; m >>= 8; p += 8; }
    c = popc32(m & 0xfu);
    if (k >= c) { k -= c; m >>= 4; p += 4; }
    c = popc32(m & 0x3u);
    if (k >= c) { k -= c; m >>= 2; p += 2; }
    c = (int)(m & 1u);
    if (k >= c) p += 1;
    return p;
}

// Run structure of a key: bits 0..31 = run starts (by position), bits 32..63 = which runs
// (by run index) are at least two residues long.
XTN_HD uint64_t key_run_info(u128 key, int L) {
    const uint32_t rs = key_run_starts(key, L);
    const uint32_t lmask = L >= 32 ? 0xffffffffu : ((1u << L) - 1u);
    const uint32_t cont = ~rs & lmask;  // positions continuing a run
    uint32_t longr = 0;
    int j = 0;
    for (uint32_t m = rs; m; m &= m - 1, j++) {
        const int p = ctz32(m);
        if ((cont >> (p + 1)) & 1u) longr |= 1u << j;
    }
    return (uint64_t)rs | ((uint64_t)longr << 32);
}

// The v-th variant (0 <= v < variant_count) of a key for d <= 2, from its run structure: a
// flat index over the run-prefix deletion sets, so variants can be produced in parallel. The
// order differs from for_each_variant; the multiset is the same. v = 0 is the key; v = 1..R
// delete the first residue of run v-1; then, for each run j in order, the pairs (first residue
// of run j, q) with q the next residue of run j (when run j is long) or the first residue of
// a later run, q ascending. Run j owns c_j = (R-1-j) + long_j pairs, so the pairs of runs
// before j number j*(R-1) - j*(j-1)/2 + (long runs before j).
XTN_HD u128 variant_at(u128 key, uint64_t info, int v) {
    if (v == 0) return key;
    const uint32_t rs = (uint32_t)info, longr = (uint32_t)(info >> 32);
    const int R = popc32(rs);
    if (v <= R) return key_del(key, select_bit(rs, v - 1));
    const int w = v - R - 1;
    // largest run j with pairs_before(j) <= w
    int lo = 0, hi = R - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int before = mid * (R - 1) - mid * (mid - 1) / 2 + popc32(longr & ((1u << mid) - 1u));
        if (before <= w) lo = mid;
        else hi = mid - 1;
    }
    const int j = lo;
    const int l = w - (j * (R - 1) - j * (j - 1) / 2 + popc32(longr & ((1u << j) - 1u)));
    const int p = select_bit(rs, j);
    const int lj = (int)((longr >> j) & 1u);
    const int q = (lj && l == 0) ? p + 1 : select_bit(rs, j + 1 + l - lj);
    return key_del(key_del(key, p), q - 1);
}

// Pairs (two-deletion variants) owned by runs 0..j-1 in variant_at's order.
XTN_HD int pairs_before_run(int j, int R, uint32_t longr) {
    return j * (R - 1) - j * (j - 1) / 2 + popc32(longr & ((1u << j) - 1u));
}

// Enumerations of a key's d <= 2 variants, by deletion positions. An emitter E provides
//   e.key(v)      item v is the key itself
//   e.run(p)      the items that follow delete residue p, the first residue of a run
//   e.single(v)   item v deletes p only
//   e.pair(v, q)  item v deletes p and q (q > p: the next residue of p's run, or the first
//                 residue of a later run)

// Positions q that pair with run j starting at p.
XTN_HD uint32_t pair_positions(uint32_t rs, uint32_t longr, uint32_t lmask, int L, int j, int p) {
    uint32_t a = rs & lmask & ~((2u << p) - 1u);
    if (p + 1 < L && ((longr >> j) & 1u)) a |= 1u << (p + 1);
    return a;
}

// Task t (0 <= t < 2*ceil(R/2)) of a key's d <= 2 variants, for parallel generation with even
// work: tasks 2j and 2j+1 share the items of runs j and R-1-j (the single deletion of each run
// and its pairs; about R+1 items together), split into two halves; task 0 also emits the key.
// (Whole run pairs per task, half as many tasks, and quarters, twice as many, both measured
// slower in the generation kernel at 10M: 7.2 and 9.2 ms against 5.6 ms.)
// Item indices v are variant_at's flat order.
template <class E>
XTN_HD void task_items(int L, uint64_t info, int d, int t, E& e) {
    const uint32_t rs = (uint32_t)info, longr = (uint32_t)(info >> 32);
    const uint32_t lmask = L >= 32 ? 0xffffffffu : ((1u << L) - 1u);
    const int R = popc32(rs);
    const bool two = d >= 2 && L >= 2;
    if (t == 0) e.key(0);
    const int jA = t >> 1, jB = R - 1 - jA;
    // items of one run: the single deletion, then its pairs in ascending q
    int wA, wB = 0;
    uint32_t allowA = 0, allowB = 0;
    const int pA = select_bit(rs, jA), pB = select_bit(rs, jB);
    if (two) allowA = pair_positions(rs, longr, lmask, L, jA, pA);
    wA = 1 + popc32(allowA);
    if (jB != jA) {
        if (two) allowB = pair_positions(rs, longr, lmask, L, jB, pB);
        wB = 1 + popc32(allowB);
    }
    const int total = wA + wB, half = total >> 1;
    const int i0 = (t & 1) ? half : 0, i1 = (t & 1) ? total : half;
    auto run_items = [&](int j, int p, uint32_t allow, int a, int b) {  // local items [a, b)
        if (a >= b) return;
        e.run(p);
        if (a == 0) {
            e.single(1 + j);
            a = 1;
        }
        uint32_t m = allow;
        for (int k = 1; k < a; k++) m &= m - 1;  // skip the pairs before item a
        const int base = 1 + R + pairs_before_run(j, R, longr) - 1;
        for (int it = a; it < b; it++) {
            e.pair(base + it, ctz32(m));
            m &= m - 1;
        }
    };
    run_items(jA, pA, allowA, i0 < wA ? i0 : wA, i1 < wA ? i1 : wA);
    if (wB) run_items(jB, pB, allowB, (i0 > wA ? i0 : wA) - wA, (i1 > wA ? i1 : wA) - wA);
}

// All d <= 2 items of a key in one pass (v counts the calls; the order is by run, not
// variant_at's).
template <class E>
XTN_HD void seq_items(int L, uint64_t info, int d, E& e) {
    e.key(0);
    if (L <= 0) return;
    const uint32_t rs = (uint32_t)info, longr = (uint32_t)(info >> 32);
    const uint32_t lmask = L >= 32 ? 0xffffffffu : ((1u << L) - 1u);
    const bool two = d >= 2 && L >= 2;
    int v = 1, j = 0;
    for (uint32_t m = rs; m; m &= m - 1, j++) {
        const int p = ctz32(m);
        e.run(p);
        e.single(v++);
        if (two)
            for (uint32_t a = pair_positions(rs, longr, lmask, L, j, p); a; a &= a - 1) e.pair(v++, ctz32(a));
    }
}

// Emitter producing variant keys: f(v, key).
template <class F>
struct KeyEmitter {
    u128 k0, v1;
    F& f;
    XTN_HD void key(int v) { f(v, k0); }
    XTN_HD void run(int p) { v1 = key_del(k0, p); }
    XTN_HD void single(int v) { f(v, v1); }
    XTN_HD void pair(int v, int q) { f(v, key_del(v1, q - 1)); }
};

// Emitter producing variant hashes from a key_table: f(v, hash), equal to key_hash of the
// variant key.
template <class F>
struct TableHashEmitter {
    const uint64_t* tab;
    uint64_t c1, s1, kp;
    F& f;
    XTN_HD TableHashEmitter(const uint64_t* t, F& fn) : tab(t), kp(0), f(fn) {
        const uint64_t PL = t[kTabKey];
        c1 = kPolyRI2 * PL;             // K[p] = r G[p] + c1
        s1 = (kPolyRI - kPolyRI2) * PL;  // single deletion = K[p] + s1
    }
    XTN_HD void key(int v) { f(v, hash_fin(tab[kTabKey])); }
    XTN_HD void run(int p) { kp = kPolyR * tab[kTabG + p] + c1; }
    XTN_HD void single(int v) { f(v, hash_fin(kp + s1)); }
    XTN_HD void pair(int v, int q) { f(v, hash_fin(kp + tab[kTabG + q])); }
};

// Task t's variants as keys: f(v, key) with v the flat index (variant_at's order).
template <class F>
XTN_HD void for_each_task_variant(u128 key, int L, uint64_t info, int d, int t, F&& f) {
    KeyEmitter<F> e{key, key, f};
    task_items(L, info, d, t, e);
}

// Task t's variants as hashes: f(v, hash).
template <class F>
XTN_HD void for_each_task_hash(const uint64_t* tab, int L, uint64_t info, int d, int t, F&& f) {
    TableHashEmitter<F> e(tab, f);
    task_items(L, info, d, t, e);
}

// All of a key's d <= 2 variants as hashes with the call count v = 0, 1, ...: f(v, hash).
template <class F>
XTN_HD void for_each_seq_hash(const uint64_t* tab, int L, uint64_t info, int d, F&& f) {
    TableHashEmitter<F> e(tab, f);
    seq_items(L, info, d, e);
}

// All of a key's d <= 2 variants as hashes: f(hash).
template <class F>
XTN_HD void for_each_hash(const uint64_t* tab, int L, uint64_t info, int d, F&& f) {
    auto g = [&](int, uint64_t h) { f(h); };
    TableHashEmitter<decltype(g)> e(tab, g);
    seq_items(L, info, d, e);
}

// Row i of a group of size s owns pairs (i, i+1..s-1); it starts at local index r(i).
XTN_HD uint64_t tri_row_start(uint64_t i, uint64_t s) { return i * (2 * s - i - 1) / 2; }

// ------------------------------------------------------------------ candidate hash set sizing
// Slots (before rounding up to a power of two) for the candidate-pair hash set of Pc candidates:
// two per candidate while that is at most kDedupWideBytes of table; above that, or when
// share_sizing is set, two per expected distinct pair, the expectation being 1.25 x
// prev_share (the previous search's distinct share; 1 for a first search) x Pc, with a floor
// of kDedupWideBytes of table (2^16 slots under share_sizing). Measured on B200: 5.56M
// candidates (1.22M distinct) take 0.12 ms with 2^24 slots and 0.17 ms with 2^22; 55M
// candidates take 2.3 ms with 2^27 slots and 1.7 ms with 2^25.
constexpr uint64_t kDedupWideBytes = uint64_t(256) << 20;

inline uint64_t dedup_first_slots(uint64_t Pc, double prev_share, bool share_sizing) {
    const double share = prev_share * 1.25 < 1.0 ? prev_share * 1.25 : 1.0;
    uint64_t want = 2 * Pc;
    if (sizeof(uint64_t) * want > kDedupWideBytes || share_sizing) {
        const uint64_t floor = share_sizing ? (uint64_t(1) << 16) : kDedupWideBytes / sizeof(uint64_t);
        const uint64_t by_share = (uint64_t)(2.0 * share * (double)Pc);
        want = by_share > floor ? by_share : floor;
    }
    return want;
}

// Slots for the rerun after an insertion ran out of probes in a table of T slots.
inline uint64_t dedup_regrow_slots(uint64_t T, uint64_t Pc) { return 4 * T > 2 * Pc ? 4 * T : 2 * Pc; }

inline uint64_t pow2_at_least(uint64_t x) {
    uint64_t t = 2;
    while (t < x) t <<= 1;
    return t;
}

// ------------------------------------------------------------------ host: sequence lengths
// Non-zero when a sequence of offs[a .. b] has a length outside 1..kMaxInputLength. No early
// exit, so that the compiler vectorises it.
inline uint32_t offsets_bad(const uint32_t* offs, int a, int b) {
    uint32_t bad = 0;
    for (int i = a; i < b; i++)
        bad |= (uint32_t)(offs[i + 1] <= offs[i]) | (uint32_t)(offs[i + 1] - offs[i] > (uint32_t)kMaxInputLength);
    return bad;
}

// The first of n sequences (offsets offs[0..n]) whose length is outside 1..kMaxInputLength, or
// -1. From 2^20 sequences on, up to `threads` (at most 4) host threads share the scan for a bad
// length: the whole-search entry point runs it while the input copies are in flight, and one
// thread took 5.5 ms for 10M offsets, longer than the 3.4 ms copy (four: about 1.5 ms). A part
// whose thread cannot be started is scanned by the calling thread; the first bad index is
// searched for sequentially, only when there is one.
inline int first_bad_offset(const uint32_t* offs, int n, int threads = 4) {
    const unsigned hw = std::thread::hardware_concurrency();
    int nt = threads < 4 ? threads : 4;
    if ((unsigned)nt > hw && hw > 0) nt = (int)hw;
    if (n < (1 << 20) || nt < 1) nt = 1;
    uint32_t bad = 0;
    if (nt == 1) {
        bad = offsets_bad(offs, 0, n);
    } else {
        uint32_t part[4] = {0, 0, 0, 0};
        std::thread th[3];
        int started = 0;  // threads 1..started run
        try {
            for (int t = 1; t < nt; t++) {
                th[t - 1] = std::thread([=, &part] {
                    part[t] = offsets_bad(offs, (int)((int64_t)n * t / nt), (int)((int64_t)n * (t + 1) / nt));
                });
                started = t;
            }
        } catch (...) {  // (no exception may leave a C entry point)
        }
        part[0] = offsets_bad(offs, 0, (int)((int64_t)n / nt));
        for (int t = 1; t < nt; t++) {
            if (t <= started) th[t - 1].join();
            else part[t] = offsets_bad(offs, (int)((int64_t)n * t / nt), (int)((int64_t)n * (t + 1) / nt));
        }
        for (int t = 0; t < nt; t++) bad |= part[t];
    }
    if (!bad) return -1;
    for (int i = 0; i < n; i++)
        if (offs[i + 1] <= offs[i] || offs[i + 1] - offs[i] > (uint32_t)kMaxInputLength) return i;
    return -1;
}

// ------------------------------------------------------------------ distances
// Levenshtein distance by Myers' bit-vector algorithm in Hyyro's global form
// (G. Myers, J. ACM 46(3) 1999; H. Hyyro, 2001). `a` is the pattern (1 <= m <= bits of W); W is
// uint32_t for patterns of up to 32 residues (one instruction per word operation instead of two)
// or uint64_t up to 64.
template <class W>
XTN_HD int lev_myers(const uint8_t* a, int m, const uint8_t* b, int n) {
    constexpr int kBits = 8 * (int)sizeof(W);
    W p0 = 0, p1 = 0, p2 = 0, p3 = 0, p4 = 0;  // bit-sliced residue codes of a
    for (int i = 0; i < m; i++) {
        unsigned c = (unsigned)code_of(a[i]);
        const W bit = (W)1 << i;
        if (c & 1u) p0 |= bit;
        if (c & 2u) p1 |= bit;
        if (c & 4u) p2 |= bit;
        if (c & 8u) p3 |= bit;
        if (c & 16u) p4 |= bit;
    }
    const W mask = m == kBits ? ~(W)0 : (W)(((W)1 << m) - 1);
    const W high = (W)1 << (m - 1);
    W pv = mask, mv = 0;
    int score = m;
    for (int j = 0; j < n; j++) {
        unsigned c = (unsigned)code_of(b[j]);
        W eq = mask;
        eq &= (c & 1u) ? p0 : (W)~p0;
        eq &= (c & 2u) ? p1 : (W)~p1;
        eq &= (c & 4u) ? p2 : (W)~p2;
        eq &= (c & 8u) ? p3 : (W)~p3;
        eq &= (c & 16u) ? p4 : (W)~p4;
        const W xv = eq | mv;
        const W xh = (W)((W)((W)(eq & pv) + pv) ^ pv) | eq;
        W ph = (W)(mv | (W)~(W)(xh | pv));
        W mh = pv & xh;
        if (ph & high) score++;
        else if (mh & high) score--;
        ph = (W)((W)(ph << 1) | (W)1);
        mh = (W)(mh << 1);
        pv = (W)(mh | (W)~(W)(xv | ph));
        mv = ph & xv;
    }
    return score;
}
XTN_HD int lev_myers64(const uint8_t* a, int m, const uint8_t* b, int n) { return lev_myers<uint64_t>(a, m, b, n); }

// Exact Levenshtein with the column held in `col` (>= m+1 ints), stopping early once every
// cell of a column exceeds `cap` (the result is then some value > cap).
XTN_HD int lev_dp(const uint8_t* a, int m, const uint8_t* b, int n, int* col, int cap) {
    for (int y = 0; y <= m; y++) col[y] = y;
    for (int x = 1; x <= n; x++) {
        int lastdiag = col[0];
        col[0] = x;
        int best = x;
        for (int y = 1; y <= m; y++) {
            int old = col[y];
            int v = col[y] + 1, w = col[y - 1] + 1, z = lastdiag + (a[y - 1] == b[x - 1] ? 0 : 1);
            int r = v < w ? v : w;
            r = r < z ? r : z;
            col[y] = r;
            lastdiag = old;
            best = best < r ? best : r;
        }
        if (best > cap) return cap + 1;
    }
    return col[m];
}

// Hamming as the reference computes it (S/src/kernel.cu:290-300): 77 for unequal
// lengths, and the mismatch count held in a signed char (wraps past 127). Also returns the
// unwrapped count through *raw.
XTN_HD int hamming_ref(const uint8_t* a, int la, const uint8_t* b, int lb, int* raw) {
    if (la != lb) {
        *raw = kHammingLenMismatch;
        return kHammingLenMismatch;
    }
    int m = 0;
    for (int i = 0; i < la; i++) m += a[i] != b[i];
    *raw = m;
    return (int)(int8_t)(uint8_t)(m & 0xFF);
}

// True when the first-18-residue keys of a and b share a deletion variant of at most d
// deletions each, i.e. when LCS(A, B) >= max(|A|, |B|) - d for the prefixes A, B. This is
// the reference's candidate condition; the verify step needs it only where the reference's
// wrapped Hamming counter accepts a pair whose true distance exceeds d.
XTN_HD bool prefixes_share_variant(const uint8_t* a, int la, const uint8_t* b, int lb, int d) {
    int A = la < kKeyLen ? la : kKeyLen, B = lb < kKeyLen ? lb : kKeyLen;
    int need = (A > B ? A : B) - d;
    if (need <= 0) return true;
    int row[kKeyLen + 1];
    for (int j = 0; j <= B; j++) row[j] = 0;
    for (int i = 1; i <= A; i++) {
        int diag = 0;
        for (int j = 1; j <= B; j++) {
            int up = row[j];
            int v = a[i - 1] == b[j - 1] ? diag + 1 : (row[j] > row[j - 1] ? row[j] : row[j - 1]);
            diag = up;
            row[j] = v;
        }
    }
    return row[B] >= need;
}

}  // namespace xtn
