// Seeded synthetic CDR3 generator for tests and benchmarks (host only, no GPU).
//
// The reference measures on subsets of the Emerson CDR3 data, which are not available
// here; these generators stand in with the shapes the workloads are defined by:
//   * lengths: discrete normal (mean 15, sd 2), clipped to 8..22;
//   * first residue 'C' and last residue 'F' with probability 0.9 each;
//   * other residues i.i.d. from a fixed skewed 20-letter distribution (top 5 = 50%);
//   * "mutant" mode: a fraction of rows are 1-2 random substitutions/insertions/deletions
//     of an earlier row;
//   * "cluster" mode: a fraction of rows sit in mutant clusters whose size is
//     2 + Geometric(0.3) capped at 50 (members are 1-2 edits from the cluster seed), a
//     fraction are exact duplicates of other rows, the rest are independent; rows are
//     shuffled;
//   * "overlap" mode: R repertoires with log-uniform sizes, a fraction of each drawn from a
//     shared pool, and a duplicate_count per row from a discrete power law of exponent 1.5
//     (P(count >= k) ~ k^-0.5) capped at 1e6.
// All randomness comes from xoshiro256** seeded through splitmix64, so a seed gives the
// same rows on every machine.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        for (int i = 0; i < 4; i++) {  // splitmix64
            seed += 0x9e3779b97f4a7c15ULL;
            uint64_t z = seed;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
            s[i] = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {  // xoshiro256** (Blackman & Vigna)
        uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uni() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t n) { return n ? next() % n : 0; }
    double normal() {
        double u1 = uni(), u2 = uni();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// Fixed skewed residue distribution: S G A T E hold 50%.
const char kRes[20] = {'S', 'G', 'A', 'T', 'E', 'Q', 'L', 'N', 'D', 'Y', 'R', 'P', 'K', 'V', 'F', 'W', 'H', 'I', 'M', 'C'};
const double kProb[20] = {0.12, 0.11, 0.10, 0.09, 0.08, 0.05, 0.048, 0.045, 0.042, 0.04,
                          0.038, 0.035, 0.033, 0.03, 0.028, 0.025, 0.022, 0.02, 0.018, 0.026};

struct Gen {
    Rng rng;
    double cum[20];
    explicit Gen(uint64_t seed) : rng(seed) {
        double c = 0;
        for (int i = 0; i < 20; i++) {
            c += kProb[i];
            cum[i] = c;
        }
        cum[19] = 1.0;
    }
    char residue() {
        double u = rng.uni();
        for (int i = 0; i < 20; i++)
            if (u < cum[i]) return kRes[i];
        return kRes[19];
    }
    int length() {
        int L = (int)std::lround(15.0 + 2.0 * rng.normal());
        return L < 8 ? 8 : (L > 22 ? 22 : L);
    }
    std::string random_seq() {
        int L = length();
        std::string s(L, 'A');
        for (int i = 0; i < L; i++) s[i] = residue();
        if (rng.uni() < 0.9) s[0] = 'C';
        if (rng.uni() < 0.9) s[L - 1] = 'F';
        return s;
    }
    std::string mutate(const std::string& src) {
        std::string s = src;
        int edits = 1 + (int)rng.below(2);
        for (int e = 0; e < edits; e++) {
            int kind = (int)rng.below(3);
            if (kind == 0 && !s.empty()) {
                size_t p = rng.below(s.size());
                char c;
                do c = residue();
                while (c == s[p]);
                s[p] = c;
            } else if (kind == 1 || s.size() <= 1) {
                size_t p = rng.below(s.size() + 1);
                s.insert(s.begin() + p, residue());
            } else {
                size_t p = rng.below(s.size());
                s.erase(s.begin() + p);
            }
        }
        return s;
    }
    int cluster_size() {
        int g = 0;
        while (rng.uni() >= 0.3 && g < 48) g++;
        return 2 + g;
    }
    int count() {  // discrete power law, P(X >= k) ~ k^-0.5, capped at 1e6
        double u = 1.0 - rng.uni();
        double x = std::floor(1.0 / (u * u));
        if (x > 1e6) x = 1e6;
        return x < 1 ? 1 : (int)x;
    }
};

struct Synth {
    std::vector<char> chars;
    std::vector<uint32_t> offs{0};
    std::vector<int32_t> freq;
    std::vector<int32_t> rep_sizes;
    void add(const std::string& s) {
        chars.insert(chars.end(), s.begin(), s.end());
        offs.push_back((uint32_t)chars.size());
    }
};

void shuffle(std::vector<std::string>& v, Rng& rng) {
    for (size_t i = v.size(); i > 1; i--) std::swap(v[i - 1], v[rng.below(i)]);
}

}  // namespace

extern "C" {

// mode 0: mutant mode (fraction a of rows are 1-2 edits of an earlier row)
// mode 1: cluster mode (fraction a in mutant clusters, fraction b exact duplicates)
void* synth_nn(uint64_t seed, int64_t n, int mode, double a, double b) {
    Gen g(seed);
    Synth* out = new Synth();
    std::vector<std::string> rows;
    rows.reserve(n);
    if (mode == 0) {
        for (int64_t i = 0; i < n; i++) {
            if (i > 0 && g.rng.uni() < a) rows.push_back(g.mutate(rows[g.rng.below(rows.size())]));
            else rows.push_back(g.random_seq());
        }
    } else {
        int64_t n_cluster = (int64_t)std::llround(a * n), n_dup = (int64_t)std::llround(b * n);
        while ((int64_t)rows.size() < n_cluster) {
            int sz = g.cluster_size();
            std::string seed_seq = g.random_seq();
            rows.push_back(seed_seq);
            for (int k = 1; k < sz && (int64_t)rows.size() < n_cluster; k++) rows.push_back(g.mutate(seed_seq));
        }
        while ((int64_t)rows.size() < n - n_dup) rows.push_back(g.random_seq());
        while ((int64_t)rows.size() < n) rows.push_back(rows[g.rng.below(rows.size())]);
        shuffle(rows, g.rng);
    }
    out->chars.reserve((size_t)n * 16);
    out->offs.reserve(n + 1);
    for (auto& s : rows) out->add(s);
    return out;
}

// R repertoires, sizes log-uniform in [min_size, max_size], fraction `shared` of each drawn
// from a common pool; within a repertoire rows are distinct.
void* synth_overlap(uint64_t seed, int R, double min_size, double max_size, double shared) {
    Gen g(seed);
    Synth* out = new Synth();
    std::vector<int64_t> sizes(R);
    int64_t total = 0;
    for (int r = 0; r < R; r++) {
        double u = g.rng.uni();
        sizes[r] = (int64_t)std::llround(std::exp(std::log(min_size) + u * (std::log(max_size) - std::log(min_size))));
        total += sizes[r];
    }
    int64_t pool_n = std::max<int64_t>(16, (int64_t)(shared * total / 4));
    std::vector<std::string> pool(pool_n);
    for (auto& s : pool) s = g.random_seq();
    out->chars.reserve((size_t)total * 16);
    for (int r = 0; r < R; r++) {
        std::vector<std::string> rows;
        rows.reserve(sizes[r]);
        std::vector<uint8_t> used(pool_n, 0);
        for (int64_t k = 0; k < sizes[r]; k++) {
            if (g.rng.uni() < shared) {
                int64_t p = (int64_t)g.rng.below(pool_n);
                if (!used[p]) {
                    used[p] = 1;
                    rows.push_back(pool[p]);
                    continue;
                }
            }
            if (!rows.empty() && g.rng.uni() < 0.1) rows.push_back(g.mutate(rows[g.rng.below(rows.size())]));
            else rows.push_back(g.random_seq());
        }
        for (auto& s : rows) {
            out->add(s);
            out->freq.push_back(g.count());
        }
        out->rep_sizes.push_back((int32_t)rows.size());
    }
    return out;
}

int64_t synth_n(void* h) { return (int64_t)static_cast<Synth*>(h)->offs.size() - 1; }
int64_t synth_total_chars(void* h) { return (int64_t)static_cast<Synth*>(h)->chars.size(); }
int32_t synth_n_reps(void* h) { return (int32_t)static_cast<Synth*>(h)->rep_sizes.size(); }
void synth_copy(void* h, char* chars, uint32_t* offs, int32_t* freq, int32_t* rep_sizes) {
    Synth* s = static_cast<Synth*>(h);
    if (chars) memcpy(chars, s->chars.data(), s->chars.size());
    if (offs) memcpy(offs, s->offs.data(), s->offs.size() * 4);
    if (freq && !s->freq.empty()) memcpy(freq, s->freq.data(), s->freq.size() * 4);
    if (rep_sizes && !s->rep_sizes.empty()) memcpy(rep_sizes, s->rep_sizes.data(), s->rep_sizes.size() * 4);
}
void synth_free(void* h) { delete static_cast<Synth*>(h); }
}

#ifdef XTN_SYNTH_MAIN
// Command-line front end (bin/xtn_synth): writes a generated workload in the xt_neighbor CLI's
// input format, so that a process can be given a workload file without loading this library.
//   xtn_synth mutants     SEED N FRAC              OUT.csv [PREFIX_N PREFIX.csv]
//   xtn_synth clusters    SEED N CLUSTER_FRAC DUP  OUT.csv [PREFIX_N PREFIX.csv]
//   xtn_synth repertoires SEED R MIN MAX SHARED    OUT.csv INFO.csv [MAX_LEN]
// OUT.csv: header line, then one sequence per line ("seq,count" for repertoires); INFO.csv:
// header line, then one repertoire size per line. PREFIX.csv holds the first PREFIX_N rows.
// MAX_LEN drops the rows longer than MAX_LEN residues (and counts the repertoires without them).
#include <cstdio>
#include <cstdlib>

static bool write_rows(const Synth* s, int64_t rows, const char* path, uint32_t max_len = 0xffffffffu) {
    FILE* f = fopen(path, "wb");
    if (!f) return false;
    const bool counts = !s->freq.empty();
    std::string buf = counts ? "cdr3,count\n" : "cdr3\n";
    for (int64_t i = 0; i < rows; i++) {
        if (s->offs[i + 1] - s->offs[i] > max_len) continue;
        buf.append(s->chars.data() + s->offs[i], s->offs[i + 1] - s->offs[i]);
        if (counts) {
            buf.push_back(',');
            buf.append(std::to_string(s->freq[i]));
        }
        buf.push_back('\n');
        if (buf.size() > (size_t(32) << 20)) {
            fwrite(buf.data(), 1, buf.size(), f);
            buf.clear();
        }
    }
    fwrite(buf.data(), 1, buf.size(), f);
    return fclose(f) == 0;
}

int main(int argc, char** argv) {
    const std::string kind = argc > 1 ? argv[1] : "";
    Synth* s = nullptr;
    int next = 0;
    if (kind == "mutants" && argc >= 6) {
        s = static_cast<Synth*>(synth_nn(strtoull(argv[2], nullptr, 10), atoll(argv[3]), 0, atof(argv[4]), 0.0));
        next = 5;
    } else if (kind == "clusters" && argc >= 7) {
        s = static_cast<Synth*>(
            synth_nn(strtoull(argv[2], nullptr, 10), atoll(argv[3]), 1, atof(argv[4]), atof(argv[5])));
        next = 6;
    } else if (kind == "repertoires" && argc >= 9) {
        s = static_cast<Synth*>(
            synth_overlap(strtoull(argv[2], nullptr, 10), atoi(argv[3]), atof(argv[4]), atof(argv[5]), atof(argv[6])));
        next = 7;
    } else {
        fprintf(stderr, "usage: xtn_synth mutants|clusters|repertoires ... (see synth.cpp)\n");
        return 1;
    }
    int64_t n = (int64_t)s->offs.size() - 1;
    const uint32_t max_len = (kind == "repertoires" && argc > next + 2) ? (uint32_t)atoi(argv[next + 2]) : 0xffffffffu;
    if (!write_rows(s, n, argv[next], max_len)) return 1;
    if (kind == "repertoires") {
        FILE* f = fopen(argv[next + 1], "wb");
        if (!f) return 1;
        fputs("size\n", f);
        int64_t row = 0, kept_total = 0;
        for (int32_t r : s->rep_sizes) {
            int32_t kept = 0;
            for (int32_t k = 0; k < r; k++, row++) kept += s->offs[row + 1] - s->offs[row] <= max_len;
            if (kept > 0) fprintf(f, "%d\n", kept);
            kept_total += kept;
        }
        n = kept_total;
        if (fclose(f) != 0) return 1;
    } else if (argc > next + 2) {
        const int64_t k = std::min<int64_t>(n, atoll(argv[next + 1]));
        if (!write_rows(s, k, argv[next + 2])) return 1;
    }
    printf("%lld\n", (long long)n);
    delete s;
    return 0;
}
#endif
