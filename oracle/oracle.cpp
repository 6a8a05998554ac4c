/*
 * CPU oracle for the XTNeighbor-streaming symmetric-deletion search.
 *
 * TEST INFRASTRUCTURE ONLY. This file restates on the CPU the algorithm of the
 * reference tool (heartnetkung/XT-neighbor, xtneighbor_streaming/src/). It is the
 * checker that the CUDA product path is compared against. Only the test suite, the
 * smoke check and the benchmark's CPU-baseline leg may load it; the product library
 * and CLI never link or call it.
 *
 * Every function cites the reference file:line it restates (paths are relative to the
 * reference project; xtneighbor_streaming/ is abbreviated S/). The stage functions
 * (orc_stream1 .. orc_stream4_overlap, orc_bin_packing_*, orc_histogram) exist so that
 * the reference's own unit-test vectors (S/test/) can pin this restatement; the
 * whole-search functions (orc_nn_search, orc_overlap_search) compose the same stages
 * without the reference's host-RAM spill streams, which change where data lives but not
 * the output (S/src/xtn.cu:311-470 only partitions the min-id space into rounds/columns
 * that are concatenated in ascending order).
 *
 * Parallelism: OpenMP across host cores (the CPU baseline reports the thread count).
 */
#include <algorithm>
#include <array>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>
#include <omp.h>
#include <parallel/algorithm>

namespace {

const int MAX_COMPRESSED_LENGTH = 18;  // S/src/xtn.h:8
const int LEVENSHTEIN = 0, HAMMING = 1;  // S/src/xtn.h:12-14

struct Int3 { uint32_t e[3]; };                       // S/src/xtn.h:19-25
struct Int2 { int32_t x, y; };                        // S/src/xtn.h:30-36
struct SeqInfo { int32_t frequency, repertoire, originalIndex; };  // S/src/xtn.h:41-45

// ---------------------------------------------------------------- codec
// S/src/codec.cu:25-38 ('A'..'Y' minus B,J,O,U,X -> 1..25)
int char_encode(int c) {
    if (c < 'A' || c > 'Y') return -1;
    if (c == 'B' || c == 'J' || c == 'O' || c == 'U' || c == 'X') return -1;
    return c - ('A' - 1);
}

inline int code_at(const Int3& v, int i) { return (v.e[i / 6] >> (27 - 5 * (i % 6))) & 0x1F; }
inline void put_code(Int3& v, int i, uint32_t c) { v.e[i / 6] |= c << (27 - 5 * (i % 6)); }

// S/src/codec.cu:43-60: first 18 residues, 6 per word, MSB first; an invalid char zeroes word 0
Int3 str_encode(const char* s) {
    Int3 a{{0, 0, 0}};
    for (int i = 0; i < MAX_COMPRESSED_LENGTH; i++) {
        char c = s[i];
        if (c == '\0' || c == '\n' || c == ',' || c == '\t') break;
        int v = char_encode(c);
        if (v < 0) { a.e[0] = 0; break; }
        put_code(a, i, (uint32_t)v);
    }
    return a;
}

// S/src/codec.cu:86-106: number of non-zero codes before the first zero slot
int len_decode(const Int3& v) {
    int n = 0;
    while (n < MAX_COMPRESSED_LENGTH && code_at(v, n) != 0) n++;
    return n;
}

// S/src/codec.cu:111-149: delete residue `pos` and shift the tail up by one slot
Int3 remove_char(const Int3& v, int pos) {
    Int3 a{{0, 0, 0}};
    int o = 0;
    for (int i = 0; i < MAX_COMPRESSED_LENGTH; i++) {
        if (i == pos) continue;
        put_code(a, o++, (uint32_t)code_at(v, i));
    }
    return a;
}

// S/src/kernel.cu:594-610 (toInt3): pack the first <=18 chars of a CSR string
Int3 to_int3(const char* s, int len) {
    Int3 a{{0, 0, 0}};
    if (len > MAX_COMPRESSED_LENGTH) len = MAX_COMPRESSED_LENGTH;
    for (int i = 0; i < len; i++) put_code(a, i, (uint32_t)(s[i] - ('A' - 1)));
    return a;
}

// S/src/kernel.cu:33-57: V = sum_{k<=min(d,L)} C(L,k)
int combination_len(const Int3& v, int d) {
    int len = len_decode(v);
    int out = 1 + len;
    if (d > 1 && len > 1) out += len * (len - 1) / 2;
    if (d > 2 && len > 2) {
        int c = len * (len - 1) / 2;
        for (int i = 3; i <= d; i++) {
            c = c * (len - i + 1) / i;
            if (c <= 0) break;
            out += c;
        }
    }
    return out;
}

// S/src/generate_combination.cu:42-141 (expand_keys*): every deletion set of at most
// min(d, L) positions, emitted in post-order: the extensions S+{q} (q > max S, q ascending)
// of a set S come before S itself, and the empty set comes last. Duplicate strings are kept.
struct Expander {
    const Int3* base; int len, depth_max;
    Int3* out; uint32_t* first_keys; int64_t n;
    int pos[MAX_COMPRESSED_LENGTH + 1];
    Int3 cur_of(int depth) const {
        // apply deletions pos[0..depth) (ascending original positions) to *base
        Int3 v = *base;
        for (int k = depth - 1; k >= 0; k--) v = remove_char(v, pos[k]);
        return v;
    }
    void emit(const Int3& v) {
        out[n] = v;
        if (first_keys) first_keys[n] = v.e[1];
        n++;
    }
    void rec(int depth, int start) {
        if (depth < depth_max)
            for (int q = start; q < len; q++) {
                pos[depth] = q;
                rec(depth + 1, q + 1);
            }
        emit(cur_of(depth));
    }
};

int64_t expand_keys(const Int3& seq, int d, Int3* out, uint32_t* first_keys) {
    Expander ex;
    ex.base = &seq;
    ex.len = len_decode(seq);
    ex.depth_max = d < ex.len ? d : ex.len;
    ex.out = out; ex.first_keys = first_keys; ex.n = 0;
    ex.rec(0, 0);
    return ex.n;
}

// S/src/cub.cu:14-27: order by entry[1], then entry[0], then entry[2]
inline bool int3_less(const Int3& a, const Int3& b) {
    if (a.e[1] != b.e[1]) return a.e[1] < b.e[1];
    if (a.e[0] != b.e[0]) return a.e[0] < b.e[0];
    return a.e[2] < b.e[2];
}
inline bool int3_eq(const Int3& a, const Int3& b) {
    return a.e[0] == b.e[0] && a.e[1] == b.e[1] && a.e[2] == b.e[2];
}
// S/src/cub.cu:29-39
inline bool int2_less(const Int2& a, const Int2& b) {
    if (a.x != b.x) return a.x < b.x;
    return a.y < b.y;
}

// S/src/cub.cu:217-246: even histogram over [lo, hi) with exact integer bin math
template <typename T>
void histogram(const T* v, int64_t n, int nbins, uint64_t lo, uint64_t hi, int32_t* out) {
    for (int i = 0; i < nbins; i++) out[i] = 0;
    uint64_t range = hi - lo;
    for (int64_t i = 0; i < n; i++) {
        uint64_t x = (uint64_t)v[i];
        if (x < lo || x >= hi) continue;
        uint64_t bin = ((x - lo) * (uint64_t)nbins) / range;
        if (bin >= (uint64_t)nbins) bin = nbins - 1;
        out[bin]++;
    }
}

// ---------------------------------------------------------------- distances
// S/src/kernel.cu:235-280: Wagner-Fischer over one column of `char` cells. For strings of
// at most 127 residues no cell leaves the signed-char range, so the int DP below is the same
// number. (Longer strings make the reference's `char` loop counters wrap and never finish;
// there the restatement returns the exact distance.)
int levenshtein(const char* a, int la, const char* b, int lb) {
    int col_stack[512];
    std::vector<int> col_heap;
    int* col = col_stack;
    if (la + 1 > 512) { col_heap.resize(la + 1); col = col_heap.data(); }
    for (int y = 0; y <= la; y++) col[y] = y;
    for (int x = 1; x <= lb; x++) {
        col[0] = x;
        int lastdiag = x - 1;
        for (int y = 1; y <= la; y++) {
            int olddiag = col[y];
            int v = col[y] + 1;
            int w = col[y - 1] + 1;
            int z = lastdiag + (a[y - 1] == b[x - 1] ? 0 : 1);
            col[y] = std::min(v, std::min(w, z));
            lastdiag = olddiag;
        }
    }
    return col[la];
}

// S/src/kernel.cu:290-300: 77 when the lengths differ; the mismatch counter is a signed
// char, so counts past 127 wrap modulo 256.
int hamming(const char* a, int la, const char* b, int lb) {
    if (la != lb) return 77;
    int m = 0;
    for (int i = 0; i < la; i++) m += (a[i] != b[i]);
    return (int)(int8_t)(uint8_t)(m & 0xFF);
}

// S/src/kernel.cu:359-392 (cal_distance, NN overload): x == y is rejected; the returned
// value is the `char` the reference stores, and the pair is kept when it is <= d.
int pair_distance(const char* chars, const uint32_t* offs, int x, int y, int measure) {
    const char* a = chars + offs[x];
    const char* b = chars + offs[y];
    int la = (int)(offs[x + 1] - offs[x]), lb = (int)(offs[y + 1] - offs[y]);
    return measure == HAMMING ? hamming(a, la, b, lb) : levenshtein(a, la, b, lb);
}

// ---------------------------------------------------------------- candidate pairs
// Stages 1-3 of S/src/xtn.cu:311-431 without the spill streams: generate every deletion
// variant (with its sequence id), sort by key, and emit (min id, max id) for every pair of
// positions inside a group of equal keys (S/src/kernel.cu:157-191). Self-pairs and
// duplicates are kept here; stage 4 removes them.
struct Rec { Int3 k; int32_t id; };

std::vector<Rec> gen_records(const Int3* keys, int n, int d, int nthreads) {
    std::vector<int64_t> offs(n + 1, 0);
    for (int i = 0; i < n; i++) offs[i + 1] = offs[i] + combination_len(keys[i], d);
    std::vector<Rec> recs(offs[n]);
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<Int3> buf;
#pragma omp for schedule(dynamic, 1024)
        for (int i = 0; i < n; i++) {
            int64_t cnt = offs[i + 1] - offs[i];
            buf.resize(cnt);
            expand_keys(keys[i], d, buf.data(), nullptr);
            for (int64_t j = 0; j < cnt; j++) recs[offs[i] + j] = Rec{buf[j], i};
        }
    }
    return recs;
}

std::vector<uint64_t> candidate_pairs(std::vector<Rec>& recs, int nthreads) {
    __gnu_parallel::sort(recs.begin(), recs.end(), [](const Rec& a, const Rec& b) {
        if (!int3_eq(a.k, b.k)) return int3_less(a.k, b.k);
        return a.id < b.id;
    });
    // group boundaries
    std::vector<int64_t> starts;
    for (int64_t i = 0; i < (int64_t)recs.size(); i++)
        if (i == 0 || !int3_eq(recs[i].k, recs[i - 1].k)) starts.push_back(i);
    starts.push_back((int64_t)recs.size());
    int64_t ng = (int64_t)starts.size() - 1;
    std::vector<int64_t> poff(ng + 1, 0);
    for (int64_t g = 0; g < ng; g++) {
        int64_t s = starts[g + 1] - starts[g];
        poff[g + 1] = poff[g] + s * (s - 1) / 2;
    }
    std::vector<uint64_t> pairs(poff[ng]);
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
    for (int64_t g = 0; g < ng; g++) {
        int64_t o = poff[g];
        for (int64_t i = starts[g]; i < starts[g + 1]; i++)
            for (int64_t j = i + 1; j < starts[g + 1]; j++) {
                uint32_t a = (uint32_t)recs[i].id, b = (uint32_t)recs[j].id;
                if (a > b) std::swap(a, b);
                pairs[o++] = ((uint64_t)a << 32) | b;
            }
    }
    return pairs;
}

void sort_unique(std::vector<uint64_t>& v) {
    __gnu_parallel::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
}

struct Result {
    std::vector<Int2> pairs;
    std::vector<int8_t> dist;
    std::vector<uint64_t> freq;
    int64_t candidates = 0, unique_candidates = 0;
};

int g_threads = 0;
int nthreads_or_default() { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

}  // namespace

extern "C" {

// ---------------------------------------------------------------- codec entry points
int orc_char_encode(int c) { return char_encode(c); }
void orc_str_encode(const char* s, uint32_t* out) {
    Int3 v = str_encode(s);
    memcpy(out, v.e, 12);
}
// S/src/codec.cu:66-81; `out` must hold 19 bytes
void orc_str_decode(const uint32_t* in, char* out) {
    Int3 v; memcpy(v.e, in, 12);
    int i = 0;
    for (; i < MAX_COMPRESSED_LENGTH; i++) {
        int c = code_at(v, i);
        if (c == 0) break;
        out[i] = (char)(('A' - 1) + c);
    }
    out[i] = '\0';
}
int orc_len_decode(const uint32_t* in) { Int3 v; memcpy(v.e, in, 12); return len_decode(v); }
void orc_remove_char(const uint32_t* in, int pos, uint32_t* out) {
    Int3 v; memcpy(v.e, in, 12);
    Int3 r = remove_char(v, pos);
    memcpy(out, r.e, 12);
}
int orc_combination_len(const uint32_t* in, int d) { Int3 v; memcpy(v.e, in, 12); return combination_len(v, d); }
// `out` holds orc_combination_len(in, d) * 3 words
int64_t orc_expand_keys(const uint32_t* in, int d, uint32_t* out, uint32_t* first_keys) {
    Int3 v; memcpy(v.e, in, 12);
    return expand_keys(v, d, reinterpret_cast<Int3*>(out), first_keys);
}
void orc_to_int3(const char* s, int len, uint32_t* out) { Int3 v = to_int3(s, len); memcpy(out, v.e, 12); }
void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void) { return nthreads_or_default(); }

int orc_levenshtein(const char* a, int la, const char* b, int lb) { return levenshtein(a, la, b, lb); }
int orc_hamming(const char* a, int la, const char* b, int lb) { return hamming(a, la, b, lb); }

// S/src/cub.cu:217-246
void orc_histogram_i32(const int32_t* v, int64_t n, int nbins, int64_t lo, int64_t hi, int32_t* out) {
    histogram(v, n, nbins, (uint64_t)lo, (uint64_t)hi, out);
}
void orc_histogram_u32(const uint32_t* v, int64_t n, int nbins, uint64_t lo, uint64_t hi, int32_t* out) {
    histogram(v, n, nbins, lo, hi, out);
}

// ---------------------------------------------------------------- stage 1
// S/src/xtn_inner.cu:329-358 (stream_handler1): variants of each packed sequence in DFS
// order, ids = carry + index, stable-sorted by Int3Comparator; histogram of entry[1] over
// [0, UINT_MAX) with `nbins` bins. Returns the number of variants; `keys_out` holds 3 words
// per variant.
int64_t orc_stream1(const uint32_t* seqs, int n, int d, int carry, int nbins,
                    uint32_t* keys_out, int32_t* ids_out, int32_t* hist_out) {
    std::vector<Rec> recs;
    std::vector<uint32_t> first;
    for (int i = 0; i < n; i++) {
        Int3 v; memcpy(v.e, seqs + 3 * i, 12);
        int c = combination_len(v, d);
        std::vector<Int3> buf(c);
        std::vector<uint32_t> fk(c);
        expand_keys(v, d, buf.data(), fk.data());
        for (int j = 0; j < c; j++) { recs.push_back(Rec{buf[j], carry + i}); first.push_back(fk[j]); }
    }
    std::stable_sort(recs.begin(), recs.end(), [](const Rec& a, const Rec& b) { return int3_less(a.k, b.k); });
    for (size_t i = 0; i < recs.size(); i++) {
        memcpy(keys_out + 3 * i, recs[i].k.e, 12);
        ids_out[i] = recs[i].id;
    }
    // the histogram runs over the unsorted first-keys buffer, which holds the same multiset
    histogram(first.data(), (int64_t)first.size(), nbins, 0, 0xFFFFFFFFull, hist_out);
    return (int64_t)recs.size();
}

// ---------------------------------------------------------------- stage 2
// S/src/xtn_inner.cu:374-414 (stream_handler2) with a bin budget large enough for one bin:
// stable sort by Int3Comparator; histogram over [0, seq_len) of the smaller id of every pair
// of positions inside a group (S/src/kernel.cu:203-223); rows cut where the key changes,
// each at most max_row elements unless a single group is larger (S/src/xtn_inner.cu:77-90).
// Returns the number of rows written to rows_out.
int orc_stream2(uint32_t* keys, int32_t* ids, int n, int seq_len, int nbins, int max_row,
                int32_t* hist_out, int32_t* rows_out) {
    std::vector<Rec> recs(n);
    for (int i = 0; i < n; i++) { memcpy(recs[i].k.e, keys + 3 * i, 12); recs[i].id = ids[i]; }
    std::stable_sort(recs.begin(), recs.end(), [](const Rec& a, const Rec& b) { return int3_less(a.k, b.k); });
    std::vector<int32_t> smaller;
    std::vector<int> group_len;
    for (int i = 0; i < n;) {
        int j = i;
        while (j < n && int3_eq(recs[j].k, recs[i].k)) j++;
        group_len.push_back(j - i);
        for (int a = i; a < j; a++)
            for (int b = a + 1; b < j; b++) smaller.push_back(std::min(recs[a].id, recs[b].id));
        i = j;
    }
    histogram(smaller.data(), (int64_t)smaller.size(), nbins, 0, (uint64_t)seq_len, hist_out);
    int nrows = 0, row = 0;
    for (int g : group_len) {
        if (row > 0 && row + g > max_row) { rows_out[nrows++] = row; row = 0; }
        row += g;
    }
    if (row > 0) rows_out[nrows++] = row;
    for (int i = 0; i < n; i++) { memcpy(keys + 3 * i, recs[i].k.e, 12); ids[i] = recs[i].id; }
    return nrows;
}

// ---------------------------------------------------------------- stage 3
// S/src/xtn_inner.cu:428-473 (stream_handler3) for sorted, grouped input and one bin:
// every pair of positions in a group whose smaller id is <= lowerbound, as (min, max),
// sorted by Int2Comparator (S/src/kernel.cu:157-191, S/src/cub.cu:116-124); histogram of
// the smaller ids over [0, seq_len); then the rows that survive the round
// (S/src/kernel.cu:501-521): ids > lowerbound in groups that keep at least two of them.
// Returns the number of pairs; *n_inout becomes the number of surviving rows.
int64_t orc_stream3(uint32_t* keys, int32_t* ids, int* n_inout, int lowerbound, int seq_len, int nbins,
                    int32_t* pairs_out, int64_t pairs_cap, int32_t* hist_out) {
    int n = *n_inout;
    std::vector<Int2> pairs;
    std::vector<int32_t> lesser;
    std::vector<uint32_t> keep_k;
    std::vector<int32_t> keep_v;
    for (int i = 0; i < n;) {
        int j = i;
        while (j < n && keys[3 * j] == keys[3 * i] && keys[3 * j + 1] == keys[3 * i + 1] &&
               keys[3 * j + 2] == keys[3 * i + 2])
            j++;
        for (int a = i; a < j; a++)
            for (int b = a + 1; b < j; b++) {
                Int2 p{std::min(ids[a], ids[b]), std::max(ids[a], ids[b])};
                if (p.x > lowerbound) continue;
                pairs.push_back(p);
                lesser.push_back(p.x);
            }
        int valid = 0;
        for (int a = i; a < j; a++) valid += ids[a] > lowerbound;
        if (valid >= 2)
            for (int a = i; a < j; a++)
                if (ids[a] > lowerbound) {
                    keep_k.insert(keep_k.end(), keys + 3 * a, keys + 3 * a + 3);
                    keep_v.push_back(ids[a]);
                }
        i = j;
    }
    std::stable_sort(pairs.begin(), pairs.end(), int2_less);
    histogram(lesser.data(), (int64_t)lesser.size(), nbins, 0, (uint64_t)seq_len, hist_out);
    int64_t np = (int64_t)pairs.size();
    for (int64_t i = 0; i < np && i < pairs_cap; i++) { pairs_out[2 * i] = pairs[i].x; pairs_out[2 * i + 1] = pairs[i].y; }
    *n_inout = (int)keep_v.size();
    memcpy(keys, keep_k.data(), keep_k.size() * 4);
    memcpy(ids, keep_v.data(), keep_v.size() * 4);
    return np;
}

// ---------------------------------------------------------------- stage 4 (NN)
// S/src/xtn_inner.cu:487-500 (stream_handler4_nn): sort + unique the pairs, verify on the
// full strings, keep dist <= d. Returns the number of output pairs.
int64_t orc_stream4_nn(const char* chars, const uint32_t* offs, int seq_len, const int32_t* pairs, int64_t np,
                       int d, int measure, int32_t* pairs_out, int8_t* dist_out) {
    std::vector<uint64_t> v(np);
    for (int64_t i = 0; i < np; i++) v[i] = ((uint64_t)(uint32_t)pairs[2 * i] << 32) | (uint32_t)pairs[2 * i + 1];
    sort_unique(v);
    int64_t m = 0;
    for (uint64_t p : v) {
        int x = (int)(p >> 32), y = (int)(uint32_t)p;
        if (x == y || x >= seq_len || y >= seq_len) continue;
        int dist = pair_distance(chars, offs, x, y, measure);
        if ((int8_t)dist > d) continue;
        pairs_out[2 * m] = x; pairs_out[2 * m + 1] = y; dist_out[m] = (int8_t)dist;
        m++;
    }
    return m;
}

// ---------------------------------------------------------------- bin packing
// S/src/xtn_inner.cu:279-315 (solve_bin_packing_offsets): row-wise cumulative histograms;
// columns assigned to bin (column total >> exponent); per row, the last cumulative value of
// each run of equal assignments. Returns the number of offsets per row (out is rows x that).
int orc_bin_packing_offsets(const int32_t* hist, int nrow, int nlevel, int exponent, int32_t* out) {
    std::vector<int64_t> cum((size_t)nrow * nlevel);
    for (int r = 0; r < nrow; r++) {
        int64_t s = 0;
        for (int c = 0; c < nlevel; c++) { s += hist[(size_t)r * nlevel + c]; cum[(size_t)r * nlevel + c] = s; }
    }
    std::vector<int64_t> assign(nlevel);
    for (int c = 0; c < nlevel; c++) {
        int64_t t = 0;
        for (int r = 0; r < nrow; r++) t += cum[(size_t)r * nlevel + c];
        assign[c] = t >> exponent;
    }
    // max-reduce-by-key over the flattened (row-major) matrix; runs may cross rows
    std::vector<int32_t> flat;
    int64_t best = 0, prev = 0;
    for (size_t i = 0; i < cum.size(); i++) {
        int64_t key = assign[i % nlevel];
        if (i == 0 || key != prev) {
            if (i > 0) flat.push_back((int32_t)best);
            best = cum[i];
        } else {
            best = std::max(best, cum[i]);
        }
        prev = key;
    }
    flat.push_back((int32_t)best);
    int len = (int)flat.size();
    if (len % nrow == 0) {
        int per = len / nrow;
        for (int i = 0; i < len; i++) out[i] = flat[i];
        return per;
    }
    if (len == 1) {
        for (int r = 0; r < nrow; r++) out[r] = (int32_t)cum[(size_t)r * nlevel + nlevel - 1];
        return 1;
    }
    return -1;
}

// S/src/xtn_inner.cu:245-267 (solve_bin_packing_lowerbounds) with S/src/kernel.cu:474-490
// (gen_bounds): column c's upper id is seq_len*(c+1)/nlevel - 1 and its key is
// (sum over rows of the row-cumulative histogram) >> exponent; the output is the max upper
// id of each run of equal keys. Returns the number of bounds.
int orc_bin_packing_lowerbounds(const int32_t* hist, int nrow, int nlevel, int seq_len, int exponent, int32_t* out) {
    std::vector<uint64_t> cum((size_t)nrow * nlevel);
    for (int r = 0; r < nrow; r++) {
        uint64_t s = 0;
        for (int c = 0; c < nlevel; c++) { s += (uint64_t)(int64_t)hist[(size_t)r * nlevel + c]; cum[(size_t)r * nlevel + c] = s; }
    }
    int n = 0;
    int64_t prev_key = -1;
    for (int c = 0; c < nlevel; c++) {
        uint64_t t = 0;
        for (int r = 0; r < nrow; r++) t += cum[(size_t)r * nlevel + c];
        int64_t key = (int64_t)(t >> exponent);
        int32_t val = (int32_t)((uint64_t)seq_len * (uint64_t)(c + 1) / (uint64_t)nlevel) - 1;
        if (c == 0 || key != prev_key) out[n++] = val;
        else out[n - 1] = std::max(out[n - 1], val);
        prev_key = key;
    }
    return n;
}

// ---------------------------------------------------------------- overlap mode
// S/src/cub.cu:55-78 (SeqInfoComparator): byte-wise, then shorter first
static bool seq_less(const char* chars, const uint32_t* offs, int a, int b) {
    int la = (int)(offs[a + 1] - offs[a]), lb = (int)(offs[b + 1] - offs[b]);
    int m = std::min(la, lb);
    int c = memcmp(chars + offs[a], chars + offs[b], (size_t)m);
    if (c != 0) return c < 0;
    return la < lb;
}
static bool seq_eq(const char* chars, const uint32_t* offs, int a, int b) {
    int la = (int)(offs[a + 1] - offs[a]), lb = (int)(offs[b + 1] - offs[b]);
    return la == lb && memcmp(chars + offs[a], chars + offs[b], (size_t)la) == 0;
}

// S/src/xtn_overlap_inner.cu:57-124 (overlap_mode_init): stable sort of SeqInfo by the full
// string, counts of equal strings (cumulative), packed keys of the unique strings, and the
// diagonal term: for occurrences i <= j of one unique string, f_i*f_j (as size_t) summed per
// (rep_i, rep_j). info is sorted in place. Returns the number of unique strings; the diagonal
// entries (rep pair + sum) are written sorted by Int2Comparator, their count to *n_diag.
int orc_overlap_init(const char* chars, const uint32_t* offs, int32_t* info /*n x 3*/, int n,
                     int32_t* cum_counts_out, uint32_t* keys_out, int32_t* diag_pairs_out, uint64_t* diag_sum_out,
                     int* n_diag) {
    std::vector<SeqInfo> si(n);
    memcpy(si.data(), info, sizeof(SeqInfo) * n);
    std::stable_sort(si.begin(), si.end(), [&](const SeqInfo& a, const SeqInfo& b) {
        return seq_less(chars, offs, a.originalIndex, b.originalIndex);
    });
    memcpy(info, si.data(), sizeof(SeqInfo) * n);
    std::map<std::pair<int, int>, uint64_t> diag;
    int u = 0, run_start = 0;
    for (int i = 1; i <= n; i++) {
        if (i == n || !seq_eq(chars, offs, si[i].originalIndex, si[run_start].originalIndex)) {
            cum_counts_out[u] = i;
            int o = si[run_start].originalIndex;
            Int3 k = to_int3(chars + offs[o], (int)(offs[o + 1] - offs[o]));
            memcpy(keys_out + 3 * u, k.e, 12);
            for (int a = run_start; a < i; a++)
                for (int b = a; b < i; b++)
                    diag[{si[a].repertoire, si[b].repertoire}] += (uint64_t)(int64_t)si[a].frequency * (uint64_t)(int64_t)si[b].frequency;
            u++;
            run_start = i;
        }
    }
    int m = 0;
    for (auto& kv : diag) {
        diag_pairs_out[2 * m] = kv.first.first;
        diag_pairs_out[2 * m + 1] = kv.first.second;
        diag_sum_out[m] = kv.second;
        m++;
    }
    *n_diag = m;
    return u;
}

// S/src/xtn_overlap_inner.cu:141-203 (stream_handler4_overlap) with S/src/kernel.cu:317-357
// (cal_distance, overlap overload) and :405-435 (pair2rep): dedup the unique-id pairs, verify
// on the strings of each unique id, and for every verified (u, v) add f_i*f_j (x2 when both
// occurrences are in the same repertoire) to (min rep, max rep). cum_counts are the
// inclusive run ends over the sorted info. Entries are written sorted; returns their count.
int orc_stream4_overlap(const char* chars, const uint32_t* offs, const int32_t* info /*sorted*/, const int32_t* cum_counts,
                        int n_unique, const int32_t* pairs, int64_t np, int d, int measure,
                        int32_t* rep_pairs_out, uint64_t* sums_out) {
    const SeqInfo* si = reinterpret_cast<const SeqInfo*>(info);
    std::vector<uint64_t> v(np);
    for (int64_t i = 0; i < np; i++) v[i] = ((uint64_t)(uint32_t)pairs[2 * i] << 32) | (uint32_t)pairs[2 * i + 1];
    sort_unique(v);
    std::map<std::pair<int, int>, uint64_t> acc;
    for (uint64_t p : v) {
        int x = (int)(p >> 32), y = (int)(uint32_t)p;
        if (x == y || x >= n_unique || y >= n_unique) continue;
        int ox = si[cum_counts[x] - 1].originalIndex, oy = si[cum_counts[y] - 1].originalIndex;
        int dist = pair_distance(chars, offs, ox, oy, measure);
        if ((int8_t)dist > d) continue;
        int s1 = x == 0 ? 0 : cum_counts[x - 1], e1 = cum_counts[x];
        int s2 = cum_counts[y - 1], e2 = cum_counts[y];
        for (int i = s1; i < e1; i++)
            for (int j = s2; j < e2; j++) {
                int ri = si[i].repertoire, rj = si[j].repertoire;
                uint64_t f = (uint64_t)(int64_t)si[i].frequency * (uint64_t)(int64_t)si[j].frequency;
                if (ri == rj) f *= 2;
                acc[{std::min(ri, rj), std::max(ri, rj)}] += f;
            }
    }
    int m = 0;
    for (auto& kv : acc) {
        rep_pairs_out[2 * m] = kv.first.first;
        rep_pairs_out[2 * m + 1] = kv.first.second;
        sums_out[m] = kv.second;
        m++;
    }
    return m;
}

// ---------------------------------------------------------------- whole searches
void* orc_result_new(void) { return new Result(); }
void orc_result_free(void* r) { delete static_cast<Result*>(r); }
int64_t orc_result_len(void* r) { return (int64_t)static_cast<Result*>(r)->pairs.size(); }
int64_t orc_result_candidates(void* r) { return static_cast<Result*>(r)->candidates; }
int64_t orc_result_unique_candidates(void* r) { return static_cast<Result*>(r)->unique_candidates; }
void orc_result_copy(void* r, int32_t* pairs_out, int8_t* dist_out, uint64_t* freq_out) {
    Result* R = static_cast<Result*>(r);
    for (size_t i = 0; i < R->pairs.size(); i++) { pairs_out[2 * i] = R->pairs[i].x; pairs_out[2 * i + 1] = R->pairs[i].y; }
    if (dist_out && !R->dist.empty()) memcpy(dist_out, R->dist.data(), R->dist.size());
    if (freq_out && !R->freq.empty()) memcpy(freq_out, R->freq.data(), R->freq.size() * 8);
}

// Nearest-neighbour mode, S/src/xtn.cu:267-473 composed from the stages above: returns
// every (x < y) whose first-18-residue keys share a <=d deletion variant and whose full
// strings are within d, sorted by (x, y), with the reference's `char` distance.
int orc_nn_search(const char* chars, const uint32_t* offs, int n, int d, int measure, void* result) {
    Result* R = static_cast<Result*>(result);
    int nt = nthreads_or_default();
    std::vector<Int3> keys(n);
#pragma omp parallel for num_threads(nt)
    for (int i = 0; i < n; i++) keys[i] = to_int3(chars + offs[i], (int)(offs[i + 1] - offs[i]));
    std::vector<Rec> recs = gen_records(keys.data(), n, d, nt);
    std::vector<uint64_t> pairs = candidate_pairs(recs, nt);
    std::vector<Rec>().swap(recs);
    R->candidates = (int64_t)pairs.size();
    sort_unique(pairs);
    R->unique_candidates = (int64_t)pairs.size();
    int64_t np = (int64_t)pairs.size();
    std::vector<int8_t> dist(np);
    std::vector<uint8_t> keep(np);
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nt)
    for (int64_t i = 0; i < np; i++) {
        int x = (int)(pairs[i] >> 32), y = (int)(uint32_t)pairs[i];
        keep[i] = 0;
        if (x == y) continue;
        int dd = pair_distance(chars, offs, x, y, measure);
        if ((int8_t)dd <= d) { keep[i] = 1; dist[i] = (int8_t)dd; }
    }
    R->pairs.clear(); R->dist.clear();
    for (int64_t i = 0; i < np; i++)
        if (keep[i]) {
            R->pairs.push_back(Int2{(int32_t)(pairs[i] >> 32), (int32_t)(uint32_t)pairs[i]});
            R->dist.push_back(dist[i]);
        }
    return 0;
}

// Overlap mode, S/src/xtn.cu:267-480 with S/src/xtn_overlap_inner.cu: info holds
// (frequency, repertoire, originalIndex) per input row. Result entries are (rep_x <= rep_y)
// sorted, with their summed count products (mod 2^64, as the reference's size_t sums).
int orc_overlap_search(const char* chars, const uint32_t* offs, int n, const int32_t* info_in, int d, int measure,
                       void* result) {
    Result* R = static_cast<Result*>(result);
    int nt = nthreads_or_default();
    std::vector<int32_t> info(info_in, info_in + 3 * (size_t)n);
    std::vector<int32_t> cum(n);
    std::map<std::pair<int, int>, uint64_t> acc;
    {
        // the same sort + dedup as orc_overlap_init
        std::vector<SeqInfo> si(n);
        memcpy(si.data(), info.data(), sizeof(SeqInfo) * n);
        __gnu_parallel::stable_sort(si.begin(), si.end(), [&](const SeqInfo& a, const SeqInfo& b) {
            return seq_less(chars, offs, a.originalIndex, b.originalIndex);
        });
        memcpy(info.data(), si.data(), sizeof(SeqInfo) * n);
    }
    const SeqInfo* si = reinterpret_cast<const SeqInfo*>(info.data());
    int u = 0, run_start = 0;
    std::vector<Int3> keys;
    for (int i = 1; i <= n; i++) {
        if (i == n || !seq_eq(chars, offs, si[i].originalIndex, si[run_start].originalIndex)) {
            cum[u] = i;
            int o = si[run_start].originalIndex;
            keys.push_back(to_int3(chars + offs[o], (int)(offs[o + 1] - offs[o])));
            for (int a = run_start; a < i; a++)
                for (int b = a; b < i; b++)
                    acc[{si[a].repertoire, si[b].repertoire}] +=
                        (uint64_t)(int64_t)si[a].frequency * (uint64_t)(int64_t)si[b].frequency;
            u++;
            run_start = i;
        }
    }
    std::vector<Rec> recs = gen_records(keys.data(), u, d, nt);
    std::vector<uint64_t> pairs = candidate_pairs(recs, nt);
    std::vector<Rec>().swap(recs);
    R->candidates = (int64_t)pairs.size();
    sort_unique(pairs);
    R->unique_candidates = (int64_t)pairs.size();
    for (uint64_t p : pairs) {
        int x = (int)(p >> 32), y = (int)(uint32_t)p;
        if (x == y) continue;
        int ox = si[cum[x] - 1].originalIndex, oy = si[cum[y] - 1].originalIndex;
        int dist = pair_distance(chars, offs, ox, oy, measure);
        if ((int8_t)dist > d) continue;
        int s1 = x == 0 ? 0 : cum[x - 1], e1 = cum[x];
        int s2 = cum[y - 1], e2 = cum[y];
        for (int i = s1; i < e1; i++)
            for (int j = s2; j < e2; j++) {
                int ri = si[i].repertoire, rj = si[j].repertoire;
                uint64_t f = (uint64_t)(int64_t)si[i].frequency * (uint64_t)(int64_t)si[j].frequency;
                if (ri == rj) f *= 2;
                acc[{std::min(ri, rj), std::max(ri, rj)}] += f;
            }
    }
    R->pairs.clear(); R->freq.clear();
    for (auto& kv : acc) {
        R->pairs.push_back(Int2{kv.first.first, kv.first.second});
        R->freq.push_back(kv.second);
    }
    return 0;
}

// Exhaustive neighbours of a few query sequences: every (min, max, dist) with the query on
// one side and dist(query, j) <= d under the verification semantics above (x != y). This is
// the reference's output restricted to those queries when every sequence is shorter than 128
// residues: there a distance <= d implies a shared deletion variant of the 18-residue keys,
// so the candidate stage of S/src/xtn.cu misses nothing. Used to check completeness on
// inputs too large for a full oracle run. Returns the number of triples (written up to cap).
int64_t orc_brute_neighbors(const char* chars, const uint32_t* offs, int n, const int32_t* queries, int nq, int d,
                            int measure, int32_t* out, int64_t cap) {
    std::vector<std::array<int32_t, 3>> all;
    const int nt = nthreads_or_default();
    for (int qi = 0; qi < nq; qi++) {
        const int q = queries[qi];
        const int lq = (int)(offs[q + 1] - offs[q]);
        std::vector<std::vector<std::array<int32_t, 3>>> part(nt);
#pragma omp parallel for schedule(static) num_threads(nt)
        for (int j = 0; j < n; j++) {
            if (j == q) continue;
            const int lj = (int)(offs[j + 1] - offs[j]);
            if (measure == LEVENSHTEIN ? std::abs(lq - lj) > d : (lq != lj && 77 > d)) continue;
            const int dist = pair_distance(chars, offs, q, j, measure);
            if (dist <= d) part[omp_get_thread_num()].push_back({std::min(q, j), std::max(q, j), dist});
        }
        for (auto& v : part) all.insert(all.end(), v.begin(), v.end());
    }
    std::sort(all.begin(), all.end());
    all.erase(std::unique(all.begin(), all.end()), all.end());
    for (int64_t i = 0; i < (int64_t)all.size() && i < cap; i++)
        for (int k = 0; k < 3; k++) out[3 * i + k] = all[i][k];
    return (int64_t)all.size();
}

}  // extern "C"

#ifdef ORACLE_MAIN
// Minimal command-line front end for timing the restatement: reads a CSV in the reference's
// input format (header, one sequence per row) and prints the pair count and wall time.
#include <chrono>
#include <string>
int main(int argc, char** argv) {
    if (argc < 3) { fprintf(stderr, "usage: %s input.csv d [hamming] [threads]\n", argv[0]); return 1; }
    FILE* f = fopen(argv[1], "r");
    if (!f) { perror("open"); return 1; }
    int d = atoi(argv[2]);
    int measure = (argc > 3 && std::string(argv[3]) == "hamming") ? HAMMING : LEVENSHTEIN;
    if (argc > 4) g_threads = atoi(argv[4]);
    std::vector<char> chars;
    std::vector<uint32_t> offs{0};
    char line[512];
    if (!fgets(line, sizeof line, f)) return 1;
    while (fgets(line, sizeof line, f)) {
        int i = 0;
        while (line[i] && line[i] != '\n' && line[i] != ',' && line[i] != '\t') chars.push_back(line[i++]);
        if (i) offs.push_back((uint32_t)chars.size());
    }
    fclose(f);
    int n = (int)offs.size() - 1;
    Result R;
    auto t0 = std::chrono::steady_clock::now();
    orc_nn_search(chars.data(), offs.data(), n, d, measure, &R);
    double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    printf("n=%d pairs=%zu candidates=%lld seconds=%.3f threads=%d\n", n, R.pairs.size(), (long long)R.candidates, s,
           nthreads_or_default());
    return 0;
}
#endif
