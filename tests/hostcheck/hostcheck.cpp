// Test helper: the library's host+device helpers (key packing, run-prefix variant
// enumeration, Myers/Hamming distances, prefix-variant test) compiled for the CPU, so the
// test suite can compare them with the oracle without a GPU. Not part of the product.
#include <cstdint>
#include <algorithm>
#include <cstring>

#include "../../xt-neighbor_b200/csrc/xtn_common.cuh"

using namespace xtn;

static u128 pack(const char* s, int L) {
    int Lk = L < kKeyLen ? L : kKeyLen;
    u128 v = 0;
    for (int j = 0; j < Lk; j++) v = key_put(v, j, (unsigned)code_of((uint8_t)s[j]));
    return v;
}

static void unpack(u128 v, char* out) {
    int i = 0;
    for (; i < kKeyLen; i++) {
        int c = key_get(v, i);
        if (!c) break;
        out[i] = (char)('A' - 1 + c);
    }
    out[i] = '\0';
}

extern "C" {

// Variants of the first 18 residues of s (length L) with at most d deletions: count, and
// when out != NULL the decoded strings (19 bytes each) and hashes.
int hc_variants(const char* s, int L, int d, char* out, uint64_t* hashes, int cap) {
    u128 key = pack(s, L);
    int Lk = L < kKeyLen ? L : kKeyLen;
    int n = 0;
    for_each_variant(key, Lk, d, [&](u128 k) {
        if (n < cap) {
            if (out) unpack(k, out + 19 * n);
            if (hashes) hashes[n] = key_hash(k);
        }
        n++;
    });
    return n;
}

// Variants by flat index v = 0..count-1 (decoded strings, 19 bytes each); d <= 2.
int hc_variants_flat(const char* s, int L, int d, char* out, int cap) {
    u128 key = pack(s, L);
    int Lk = L < kKeyLen ? L : kKeyLen;
    int n = variant_count(key, Lk, d);
    const uint64_t info = key_run_info(key, Lk);
    for (int v = 0; v < n && v < cap; v++) unpack(variant_at(key, info, v), out + 19 * v);
    return n;
}

// 1 when the staged scatter's tasks (for_each_task_variant, t < 2*ceil(R/2)) produce every
// flat variant index exactly once, each with variant_at's value.
int hc_task_variants_ok(const char* s, int L, int d) {
    u128 key = pack(s, L);
    int Lk = L < kKeyLen ? L : kKeyLen;
    const int n = variant_count(key, Lk, d);
    const uint64_t info = key_run_info(key, Lk);
    const int R = popc32((uint32_t)info), T = 2 * ((R + 1) / 2);
    int seen[1024] = {0};
    bool ok = n <= 1024;
    for (int t = 0; t < T && ok; t++)
        for_each_task_variant(key, Lk, info, d, t, [&](int v, u128 k) {
            if (v < 0 || v >= n || k != variant_at(key, info, v)) ok = false;
            else seen[v]++;
        });
    for (int v = 0; v < n && ok; v++) ok = seen[v] == 1;
    return ok ? 1 : 0;
}

// 1 when the key-table hashes equal key_hash of the variant keys: per task with the flat
// index (for_each_task_hash), and as a whole multiset (for_each_hash); d <= 2.
int hc_table_hash_ok(const char* s, int L, int d) {
    u128 key = pack(s, L);
    int Lk = L < kKeyLen ? L : kKeyLen;
    const int n = variant_count(key, Lk, d);
    const uint64_t info = key_run_info(key, Lk);
    uint64_t tab[kTabLen];
    key_table(key, [&](int slot, uint64_t x) { tab[slot] = x; });
    const int R = popc32((uint32_t)info), T = 2 * ((R + 1) / 2);
    int seen[1024] = {0};
    bool ok = n <= 1024;
    for (int t = 0; t < T && ok; t++)
        for_each_task_hash(tab, Lk, info, d, t, [&](int v, uint64_t h) {
            if (v < 0 || v >= n || h != key_hash(variant_at(key, info, v))) ok = false;
            else seen[v]++;
        });
    for (int v = 0; v < n && ok; v++) ok = seen[v] == 1;
    uint64_t a[1024], b[1024];
    int na = 0, nb = 0;
    for_each_hash(tab, Lk, info, d, [&](uint64_t h) { if (na < 1024) a[na++] = h; });
    for_each_variant(key, Lk, d, [&](u128 k) { if (nb < 1024) b[nb++] = key_hash(k); });
    if (na != n || nb != n) return 0;
    std::sort(a, a + na);
    std::sort(b, b + nb);
    for (int i = 0; i < n && ok; i++) ok = a[i] == b[i];
    return ok ? 1 : 0;
}

uint64_t hc_key_hash(const char* s, int L) { return key_hash(pack(s, L)); }

int hc_variant_count(const char* s, int L, int d) {
    int Lk = L < kKeyLen ? L : kKeyLen;
    return variant_count(pack(s, L), Lk, d);
}

void hc_key_del(const char* s, int L, int p, char* out) { unpack(key_del(pack(s, L), p), out); }

int hc_lev_myers(const char* a, int la, const char* b, int lb) {
    return lev_myers64((const uint8_t*)a, la, (const uint8_t*)b, lb);
}

int hc_first_bad_offset(const uint32_t* offs, int n, int threads) { return first_bad_offset(offs, n, threads); }

int hc_lev_myers32(const char* a, int la, const char* b, int lb) {
    return lev_myers<uint32_t>((const uint8_t*)a, la, (const uint8_t*)b, lb);
}

int hc_lev_dp(const char* a, int la, const char* b, int lb, int cap) {
    int col[kMaxInputLength + 2];
    return lev_dp((const uint8_t*)a, la, (const uint8_t*)b, lb, col, cap);
}

int hc_hamming(const char* a, int la, const char* b, int lb, int* raw) {
    return hamming_ref((const uint8_t*)a, la, (const uint8_t*)b, lb, raw);
}

int hc_share_variant(const char* a, int la, const char* b, int lb, int d) {
    return prefixes_share_variant((const uint8_t*)a, la, (const uint8_t*)b, lb, d) ? 1 : 0;
}

uint64_t hc_tri_row_start(uint64_t i, uint64_t s) { return tri_row_start(i, s); }
}

extern "C" {

// The candidate hash set's sizing rule (table slots after the power-of-two rounding).
uint64_t hc_dedup_first_table(uint64_t Pc, double prev_share, int share_sizing) {
    return pow2_at_least(dedup_first_slots(Pc, prev_share, share_sizing != 0));
}

uint64_t hc_dedup_regrow_table(uint64_t T, uint64_t Pc) { return pow2_at_least(dedup_regrow_slots(T, Pc)); }

}  // extern "C"
