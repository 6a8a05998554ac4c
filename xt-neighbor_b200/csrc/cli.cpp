// xt_neighbor: drop-in command-line front end over the xtn_b200 C ABI.
//
// Restates the reference CLI (S/src/cli.cu, S/src/airr.cu): the same flags, help and
// version text, input formats, validation messages on stderr ("Error: ..." via
// S/src/util.cu:13-22), exit codes (SUCCESS 0, ERROR 1, EXIT 2 for -v/-h; S/src/xtn.h:93)
// and output lines ("%d %d %d\n" for pairs, "%d %d %'lu\n" for overlap sums,
// S/src/cli.cu:199-215). Input files are read the way the reference reads them: in
// fgets() pieces of at most 499 (CSV) or 4999 (AIRR) characters, so a longer physical
// line is split into several logical lines exactly as there.
//
// Deliberate differences, where the reference's behaviour is undefined:
//   * a data line whose sequence field is empty is an error here ("input parsing error"),
//     where the reference counts the row but stores no sequence and then reads past its
//     sequence store;
//   * an AIRR header without a cdr3_aa (or, in overlap mode, duplicate_count) column is an
//     error here, where the reference indexes its column table at -1;
//   * a negative -n/-N is rejected like 0;
//   * CUDA failures exit with status 1 (the reference prints them and continues).
#include <algorithm>
#include <chrono>
#include <thread>
#include <cerrno>
#include <climits>
#include <clocale>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/xtn_b200.h"

namespace {

enum { SUCCESS = 0, ERROR = 1, EXIT = 2 };

const char kVersion[] = "2.0.0\n";  // S/src/cli.cu:9
// S/src/cli.cu:10-27
const char kHelp[] =
    "xt_neighbor: perform either nearest neighbor search for CDR3 sequences or immune repertoire overlap using "
    "GPU-based xt_neighbor algorithm.\n"
    "\t====================\n\t Common Options\n\t====================\n"
    "\t -d or --distance [number]: distance threshold defining the neighbor (default to 1)\n"
    "\t -o or --output-path [str]: path of the output file (default to no output)\n"
    "\t -m or --measurement [leven|hamming]: distance measurement (default to leven)\n"
    "\t -v or --version: print the version of the program then exit\n"
    "\t -h or --help: print the help text of the program then exit\n"
    "\t -V or --verbose: print extra detail as the program runs for debugging purpose\n"
    "\t -a or --airr: use AIRR format for input-path instead. Relevant fields are cdr3_aa and duplicate_count\n"
    "\t====================\n\t Nearest Neighbor Options\n\t====================\n"
    "\t -i or --input-path [str] (required): path of csv input file containing exactly 1 column: CDR3 amino acid "
    "sequences\n"
    "\t -n or --input-length [number] (required): number of rows given in the input file\n"
    "\t====================\n\t Repertoire Overlap Options\n\t====================\n"
    "\t -i or --input-path [str] (required): path of csv input file containing exactly 2 columns: CDR3 amino acid "
    "sequences and their frequency. Note that the sequences are assumed to be unique\n"
    "\t -n or --input-length [number] (required): number of sequences given in the input file\n"
    "\t -I or --info-path [str] (required): path of csv input file containing exactly 1 column: repertoire sizes. "
    "Note that the order of input sequence must be sorted according to this repertoire info\n"
    "\t -N or --info-length [number] (required): number of repertoires given in the info file\n";

struct Args {  // XTNArgs, S/src/xtn.h:50-60
    int distance = 1;
    int verbose = 0;
    const char* seqPath = nullptr;
    int seqLen = 0;
    const char* outputPath = nullptr;
    int measure = XTN_LEVENSHTEIN;
    const char* infoPath = nullptr;
    int infoLen = 0;
    int airr = 0;
};

int print_err(const char* s) {  // S/src/util.cu:13-16
    fprintf(stderr, "Error: %s\n", s);
    return ERROR;
}
int print_err_line(const char* s, int line) {  // S/src/util.cu:18-22
    fprintf(stderr, "Error: %s\n", s);
    fprintf(stderr, "Error line: %d\n", line);
    return ERROR;
}

// S/src/cli.cu:29-89. A flag that expects a value and is last on the line reads argv[argc],
// which is NULL; this is reported as a missing value instead of crashing.
int parse_args(int argc, char** argv, Args* a) {
    for (int i = 1; i < argc; i++) {
        const char* cur = argv[i];
        auto next = [&](const char** out) -> bool {
            if (i + 1 >= argc) return false;
            *out = argv[++i];
            return true;
        };
        const char* v = nullptr;
        if (!strcmp(cur, "-v") || !strcmp(cur, "--version")) {
            printf("%s", kVersion);
            return EXIT;
        } else if (!strcmp(cur, "-h") || !strcmp(cur, "--help")) {
            printf("%s", kHelp);
            return EXIT;
        } else if (!strcmp(cur, "-V") || !strcmp(cur, "--verbose")) {
            a->verbose = 1;
        } else if (!strcmp(cur, "-a") || !strcmp(cur, "--airr")) {
            a->airr = 1;
        } else if (!strcmp(cur, "-i") || !strcmp(cur, "--input-path")) {
            if (!next(&a->seqPath)) return print_err("missing path for seq");
        } else if (!strcmp(cur, "-I") || !strcmp(cur, "--info-path")) {
            if (!next(&a->infoPath)) return print_err("repertiore path or repertoire count is missing in overlap mode");
        } else if (!strcmp(cur, "-o") || !strcmp(cur, "--output-path")) {
            if (!next(&a->outputPath)) return print_err("output file opening failed");
        } else if (!strcmp(cur, "-d") || !strcmp(cur, "--distance")) {
            if (!next(&v)) return print_err("distance must be a valid number larger than 0");
            a->distance = atoi(v);
            if (a->distance < 1) return print_err("distance must be a valid number larger than 0");
        } else if (!strcmp(cur, "-n") || !strcmp(cur, "--input-length")) {
            if (!next(&v)) return print_err("invalid input length");
            a->seqLen = atoi(v);
            if (a->seqLen <= 0) return print_err("invalid input length");
        } else if (!strcmp(cur, "-N") || !strcmp(cur, "--info-length")) {
            if (!next(&v)) return print_err("invalid info length");
            a->infoLen = atoi(v);
            if (a->infoLen <= 0) return print_err("invalid info length");
        } else if (!strcmp(cur, "-m") || !strcmp(cur, "--measurement")) {
            if (!next(&v)) return print_err("invalid measure option");
            if (!strcmp(v, "leven")) a->measure = XTN_LEVENSHTEIN;
            else if (!strcmp(v, "hamming")) a->measure = XTN_HAMMING;
            else return print_err("invalid measure option");
        } else {
            return print_err("unknown option");
        }
    }
    if (a->seqPath == nullptr) return print_err("missing path for seq");
    if (a->seqLen == 0) return print_err("missing length for seq");
    if ((a->infoPath == nullptr) != (a->infoLen == 0))
        return print_err("repertiore path or repertoire count is missing in overlap mode");
    return SUCCESS;
}

// Reads a file in the pieces fgets(buf, size, f) would return.
class PieceReader {
   public:
    PieceReader(FILE* f, int size) : f_(f), max_(size - 1), buf_(1 << 22), line_(size + 1) {}
    // Returns false at end of file; otherwise line() holds the piece, NUL-terminated.
    bool next() {
        int n = 0;
        while (n < max_) {
            if (pos_ == end_) {
                end_ = fread(buf_.data(), 1, buf_.size(), f_);
                pos_ = 0;
                if (end_ == 0) break;
            }
            char c = buf_[pos_++];
            line_[n++] = c;
            if (c == '\n') break;
        }
        line_[n] = '\0';
        len_ = n;
        return n > 0;
    }
    char* line() { return line_.data(); }
    int len() const { return len_; }

   private:
    FILE* f_;
    int max_;
    std::vector<char> buf_;
    size_t pos_ = 0, end_ = 0;
    std::vector<char> line_;
    int len_ = 0;
};

// S/src/codec.cu:25-38
int char_encode(char c) {
    if (c < 'A' || c > 'Y') return -1;
    switch (c) {
        case 'B': case 'J': case 'O': case 'U': case 'X': return -1;
        default: return c - ('A' - 1);
    }
}

// CSR sequence store; SeqArray (S/src/codec.cu:168-243).
struct SeqStore {
    std::vector<char> chars;
    std::vector<uint32_t> offsets{0};
    int maxSize = 0;
    int size() const { return (int)offsets.size() - 1; }
    // S/src/codec.cu:175-196; returns SUCCESS, ERROR (after printing), or -1 for an empty field
    int append(const char* s) {
        if (size() >= maxSize) return print_err("SeqArray exceeding max length");
        int i = 0;
        while (i < 500) {
            char c = s[i];
            if (c == '\0' || c == '\n' || c == ',' || c == '\t') break;
            i++;
            if (char_encode(c) == -1) {
                chars.resize(offsets.back());
                return print_err("invalid char");
            }
            chars.push_back(c);
        }
        if (i == 0) return -1;
        offsets.push_back(offsets.back() + (uint32_t)i);
        return SUCCESS;
    }
};

bool blank_line(const char* s) { return !strcmp(s, "\n") || !strcmp(s, " \n"); }

bool parse_int_field(const char* s, int* out) {
    long t = strtol(s, nullptr, 10);
    if (t == 0 || t > INT_MAX || t < INT_MIN) return false;
    *out = (int)t;
    return true;
}

// One fgets()-sized piece of the input: [begin, begin + len) of the file image.
struct Piece {
    size_t begin;
    int len;
};

// Cuts file bytes [from, to) into the pieces fgets(buf, size, f) would return (a piece ends
// after a newline or after size - 1 characters). `from` must be the start of a physical line
// (or of the file), so that pieces of different segments never straddle.
static void cut_pieces(const char* data, size_t from, size_t to, int size, std::vector<Piece>* out) {
    const int maxp = size - 1;
    size_t i = from;
    while (i < to) {
        const void* nl = memchr(data + i, '\n', std::min<size_t>(to - i, (size_t)maxp));
        const size_t e = nl ? (size_t)((const char*)nl - data) + 1 : std::min(to, i + (size_t)maxp);
        out->push_back(Piece{i, (int)(e - i)});
        i = e;
    }
}

// A piece as the C string fgets() leaves: it ends at the first NUL byte, if any.
static int c_len(const char* s, int len) {
    const void* z = memchr(s, '\0', (size_t)len);
    return z ? (int)((const char*)z - s) : len;
}

// The reference skips the lines "\n" and " \n" (S/src/cli.cu:113-114).
static bool blank_piece(const char* s, int len) {
    len = c_len(s, len);
    return (len == 1 && s[0] == '\n') || (len == 2 && s[0] == ' ' && s[1] == '\n');
}

// Outcome of a data piece (a non-blank piece after the header).
enum PieceCheck { P_OK = 0, P_BAD_CHAR, P_EMPTY, P_NO_COMMA, P_BAD_NUMBER };

// SeqArray::append (S/src/codec.cu:175-196) and the frequency field (S/src/cli.cu:122-137) of
// one piece, without storing: the residues count, their validity, the frequency.
static PieceCheck check_piece(const char* s, int len, bool doubleCol, int* seq_len, int* freq) {
    len = c_len(s, len);
    int i = 0;
    while (i < 500 && i < len) {
        const char c = s[i];
        if (c == '\n' || c == ',' || c == '\t') break;
        i++;
        if (char_encode(c) == -1) return P_BAD_CHAR;
    }
    *seq_len = i;
    if (i == 0) return P_EMPTY;
    if (doubleCol) {
        const void* comma = memchr(s, ',', (size_t)len);
        if (!comma) return P_NO_COMMA;
        char num[512];
        const char* c1 = (const char*)comma + 1;
        const int m = (int)(s + len - c1);
        memcpy(num, c1, (size_t)m);
        num[m] = '\0';
        if (!parse_int_field(num, freq)) return P_BAD_NUMBER;
    }
    return P_OK;
}

// S/src/cli.cu:101-147, read in parallel. The file is loaded whole, cut into segments at
// physical line starts, and each segment into fgets() pieces (so a line longer than 499
// characters becomes several logical lines, as in the reference); the pieces are checked and
// stored by several threads. The outcome is the sequential one: the first failing piece in
// file order decides the message and its line number, and the row-count limit (-n) applies
// at the data piece where a sequential reader would reach it.
int parse_input(const char* path, SeqStore* seqs, std::vector<xtn_seq_info>* info, int len, bool doubleCol) {
    FILE* f = fopen(path, "r");
    if (!f) return print_err("input file reading failed");
    std::vector<char> data;
    {
        // one read of the whole file when its size is known (a regular file), else in pieces
        size_t size = 0;
        if (fseek(f, 0, SEEK_END) == 0) {
            const long e = ftell(f);
            if (e > 0) size = (size_t)e;
            fseek(f, 0, SEEK_SET);
        }
        data.resize(size);
        size_t got = size ? fread(data.data(), 1, size, f) : 0;
        data.resize(got);
        char buf[1 << 16];
        size_t k;
        while ((k = fread(buf, 1, sizeof buf, f)) > 0) data.insert(data.end(), buf, buf + k);
    }
    fclose(f);
    // the header is the first piece
    std::vector<Piece> head;
    cut_pieces(data.data(), 0, std::min<size_t>(data.size(), 499), 500, &head);
    const size_t body = head.empty() ? 0 : head[0].len;
    unsigned nt = std::thread::hardware_concurrency();
    nt = std::max(1u, std::min(nt, 32u));
    if (data.size() - body < (size_t(1) << 20)) nt = 1;
    // segment bounds at physical line starts
    std::vector<size_t> cut(nt + 1, data.size());
    cut[0] = body;
    for (unsigned t = 1; t < nt; t++) {
        size_t at = body + (data.size() - body) * t / nt;
        at = std::max(at, cut[t - 1]);
        while (at < data.size() && at > body && data[at - 1] != '\n') at++;
        cut[t] = at;
    }
    struct Seg {
        std::vector<Piece> pieces;
        std::vector<int> lens, freqs;  // per data piece
        size_t chars = 0;
        int64_t first_bad = -1;        // index into pieces of the first failing data piece
        PieceCheck why = P_OK;
        int64_t data_before_bad = 0;   // data pieces before it
    };
    std::vector<Seg> seg(nt);
    auto work = [&](unsigned t) {
        Seg& g = seg[t];
        cut_pieces(data.data(), cut[t], cut[t + 1], 500, &g.pieces);
        for (size_t k = 0; k < g.pieces.size(); k++) {
            const char* s = data.data() + g.pieces[k].begin;
            const int pl = g.pieces[k].len;
            if (blank_piece(s, pl)) continue;
            int sl = 0, fq = 0;
            const PieceCheck r = check_piece(s, pl, doubleCol, &sl, &fq);
            if (r != P_OK) {
                g.first_bad = (int64_t)k;
                g.why = r;
                g.data_before_bad = (int64_t)g.lens.size();
                return;
            }
            g.lens.push_back(sl);
            if (doubleCol) g.freqs.push_back(fq);
            g.chars += (size_t)sl;
        }
    };
    {
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; t++) th.emplace_back(work, t);
        work(0);
        for (auto& x : th) x.join();
    }
    // sequential outcome: walk the segments in file order. A data piece first meets the row
    // limit (SeqArray::append refuses the (len + 1)-th row), then its own checks.
    int64_t count = 0, pieces_before = 0;
    for (unsigned t = 0; t < nt; t++) {
        const Seg& g = seg[t];
        const int64_t room = (int64_t)len - count;
        const int64_t ndata = g.first_bad >= 0 ? g.data_before_bad + 1 : (int64_t)g.lens.size();
        if (ndata > room) {  // the limit is met at this segment's data piece number `room`
            int64_t seen = 0;
            for (size_t k = 0; k < g.pieces.size(); k++) {
                if (blank_piece(data.data() + g.pieces[k].begin, g.pieces[k].len)) continue;
                if (seen++ == room) {
                    print_err("SeqArray exceeding max length");
                    return print_err_line("input parsing error", (int)(2 + pieces_before + (int64_t)k));
                }
            }
        }
        if (g.first_bad >= 0) {
            const int line = (int)(2 + pieces_before + g.first_bad);
            switch (g.why) {
                case P_BAD_CHAR:
                    print_err("invalid char");
                    return print_err_line("input parsing error", line);
                case P_EMPTY: return print_err_line("input parsing error", line);
                case P_NO_COMMA: return print_err_line("input parsing error (comma expected)", line);
                default: return print_err_line("input parsing error (invalid number)", line);
            }
        }
        pieces_before += (int64_t)g.pieces.size();
        count += (int64_t)g.lens.size();
    }
    if (count != len) return print_err("input length doesn't match with the actual");
    // store: offsets by a prefix over the segments, characters copied by the threads
    size_t total = 0;
    std::vector<size_t> char_base(nt), row_base(nt);
    int64_t rows = 0;
    for (unsigned t = 0; t < nt; t++) {
        char_base[t] = total;
        row_base[t] = (size_t)rows;
        total += seg[t].chars;
        rows += (int64_t)seg[t].lens.size();
    }
    seqs->chars.resize(total);
    seqs->offsets.resize((size_t)rows + 1);
    seqs->offsets[0] = 0;
    auto store = [&](unsigned t) {
        const Seg& g = seg[t];
        size_t c = char_base[t], row = row_base[t], di = 0;
        for (size_t k = 0; k < g.pieces.size(); k++) {
            const char* s = data.data() + g.pieces[k].begin;
            if (blank_piece(s, g.pieces[k].len)) continue;
            const int sl = g.lens[di];
            memcpy(seqs->chars.data() + c, s, (size_t)sl);
            c += (size_t)sl;
            seqs->offsets[row + 1] = (uint32_t)c;
            if (doubleCol && row < info->size()) (*info)[row].frequency = g.freqs[di];
            row++;
            di++;
        }
    };
    {
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; t++) th.emplace_back(store, t);
        store(0);
        for (auto& x : th) x.join();
    }
    return SUCCESS;
}

// S/src/cli.cu:152-193
int parse_info(const char* path, std::vector<xtn_seq_info>* info, int len, int seqLen) {
    FILE* f = fopen(path, "r");
    if (!f) return print_err("info file reading failed");
    PieceReader rd(f, 500);
    int lineNumber = 1, count = 0, idx = 0;
    rd.next();
    while (rd.next()) {
        lineNumber++;
        char* line = rd.line();
        if (blank_line(line)) continue;
        long t = strtol(line, nullptr, 10);
        if (t == 0 || t > INT_MAX || t < INT_MIN) {
            fclose(f);
            return print_err_line("info parsing error (invalid number)", lineNumber);
        }
        if (idx + t > seqLen) {
            fclose(f);
            return print_err("total repertoires' size does not match sequence count [1]");
        }
        for (long k = 0; k < t; k++) {
            (*info)[idx].repertoire = count;
            (*info)[idx].original_index = idx;
            idx++;
        }
        count++;
    }
    fclose(f);
    if (count != len) return print_err("info length doesn't match with the actual");
    if (idx != seqLen) return print_err("total repertoires' size does not match sequence count [2]");
    return SUCCESS;
}

// S/src/airr.cu:24-36: offsets of the tab-separated fields, at most `ncol`
int split_offset(const char* s, std::vector<int>& off, int ncol) {
    off.assign(1, 0);
    int i = 0, count = 1;
    char c;
    while ((c = s[i++]) != '\0') {
        if (c == '\t') {
            off.push_back(i);
            if (++count == ncol) return count;
        }
    }
    return count;
}

// S/src/airr.cu:41-49
int find_idx(const char* hay, const char* needle, const std::vector<int>& off, int n) {
    const char* p = strstr(hay, needle);
    if (!p) return -1;
    int at = (int)(p - hay);
    for (int i = 0; i < n; i++)
        if (off[i] == at) return i;
    return -1;
}

// S/src/airr.cu:116-151 with extract_data (:71-104)
int parse_airr_input(const char* path, SeqStore* seqs, std::vector<xtn_seq_info>* info, int len, bool doubleCol) {
    FILE* f = fopen(path, "r");
    if (!f) return print_err("input file reading failed");
    PieceReader rd(f, 5000);
    int lineNumber = -1, count = 0;
    std::vector<int> off;
    rd.next();
    int ncol = split_offset(rd.line(), off, 300);
    int cdrIdx = find_idx(rd.line(), "cdr3_aa", off, ncol);
    int freqIdx = doubleCol ? find_idx(rd.line(), "duplicate_count", off, ncol) : -1;
    if (cdrIdx < 0 || (doubleCol && freqIdx < 0)) {
        fclose(f);
        return print_err("AIRR header lacks a required column");
    }
    while (rd.next()) {
        lineNumber++;
        char* line = rd.line();
        if (blank_line(line)) continue;
        int n = split_offset(line, off, ncol);
        bool ok = n > cdrIdx;
        if (ok) {
            int r = seqs->append(line + off[cdrIdx]);
            if (r == ERROR) {
                print_err_line("invalid seq", lineNumber);
                ok = false;
            } else if (r != SUCCESS) {
                ok = false;
            }
        }
        if (ok && doubleCol) {
            int v;
            if (n <= freqIdx) ok = false;
            else if (!parse_int_field(line + off[freqIdx], &v)) {
                print_err_line("invalid number", lineNumber);
                ok = false;
            } else if (count < (int)info->size()) {
                (*info)[count].frequency = v;
            }
        }
        if (!ok) {
            fclose(f);
            return print_err_line("line parsing error", lineNumber);
        }
        count++;
    }
    fclose(f);
    if (count != len) return print_err("input length doesn't match with the actual");
    return SUCCESS;
}

// S/src/util.cu:40-51
void print_args(const Args& a) {
    auto str = [](const char* s) { return s ? s : "(null)"; };
    printf("XTNArgs{\n");
    printf("\tdistance: %d\n", a.distance);
    printf("\tverbose: %d\n", a.verbose);
    printf("\tseqLen: %'d\n", a.seqLen);
    printf("\tseqPath: \"%s\"\n", str(a.seqPath));
    printf("\toutputPath: \"%s\"\n", str(a.outputPath));
    printf("\tmeasure: \"%s\"\n", a.measure == XTN_LEVENSHTEIN ? "leven" : "hamming");
    printf("\tinfoPath: \"%s\"\n", str(a.infoPath));
    printf("\tinfoLen: %'d\n", a.infoLen);
    printf("}\n");
}

struct Sink {
    FILE* out = nullptr;
    size_t total = 0;
    std::vector<char> buf;
    bool failed = false;
};

char* put_int(char* p, long long v) {
    char tmp[24];
    int n = 0;
    bool neg = v < 0;
    unsigned long long u = neg ? (unsigned long long)(-(v + 1)) + 1 : (unsigned long long)v;
    do {
        tmp[n++] = (char)('0' + u % 10);
        u /= 10;
    } while (u);
    if (neg) *p++ = '-';
    while (n) *p++ = tmp[--n];
    return p;
}

// file_handler_nn, S/src/cli.cu:199-206
void nn_handler(const xtn_output* o, void* user) {
    Sink* s = static_cast<Sink*>(user);
    s->total += (size_t)o->len;
    if (!s->out) return;
    const size_t kFlush = 1 << 22;
    if (s->buf.size() < kFlush + 64) s->buf.resize(kFlush + 64);
    char* p = s->buf.data();
    for (int64_t i = 0; i < o->len; i++) {
        p = put_int(p, o->index_pairs[i].x);
        *p++ = ' ';
        p = put_int(p, o->index_pairs[i].y);
        *p++ = ' ';
        p = put_int(p, o->pairwise_distances[i]);
        *p++ = '\n';
        if ((size_t)(p - s->buf.data()) >= kFlush) {
            if (fwrite(s->buf.data(), 1, p - s->buf.data(), s->out) != (size_t)(p - s->buf.data())) s->failed = true;
            p = s->buf.data();
        }
    }
    size_t n = (size_t)(p - s->buf.data());
    if (n && fwrite(s->buf.data(), 1, n, s->out) != n) s->failed = true;
}

// file_handler_overlap, S/src/cli.cu:208-215 (thousands grouping follows the locale)
void overlap_handler(const xtn_output* o, void* user) {
    Sink* s = static_cast<Sink*>(user);
    s->total += (size_t)o->len;
    if (!s->out) return;
    for (int64_t i = 0; i < o->len; i++)
        fprintf(s->out, "%d %d %'lu\n", o->index_pairs[i].x, o->index_pairs[i].y,
                (unsigned long)o->pairwise_frequencies[i]);
}

}  // namespace

// Host time since t0 in milliseconds (the -V stage breakdown).
static double ms_since(const std::chrono::steady_clock::time_point& t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

int main(int argc, char** argv) {
    const auto t_main = std::chrono::steady_clock::now();
    Args args;
    setlocale(LC_ALL, "");
    int rc = parse_args(argc, argv, &args);
    if (rc != SUCCESS) return rc;

    // CUDA start-up (device selection, context, streams) runs on its own thread while the
    // input is parsed; its outcome is looked at only once parsing has succeeded
    xtn_context* ctx = nullptr;
    int ctx_rc = XTN_SUCCESS;
    double t_init_done = 0;
    std::string init_err;  // the library's error text is per thread
    std::thread init([&] {
        ctx_rc = xtn_context_create(0, &ctx);
        if (ctx_rc != XTN_SUCCESS) init_err = xtn_last_error();
        t_init_done = ms_since(t_main);
    });
    struct Joiner {
        std::thread& t;
        xtn_context*& c;
        ~Joiner() {
            if (t.joinable()) t.join();
            xtn_context_destroy(c);
        }
    } joiner{init, ctx};

    bool overlap = args.infoPath != nullptr;
    SeqStore seqs;
    seqs.maxSize = args.seqLen;
    seqs.chars.reserve((size_t)args.seqLen * 18);
    seqs.offsets.reserve((size_t)args.seqLen + 1);
    std::vector<xtn_seq_info> info;
    if (overlap) {
        info.assign(args.seqLen, xtn_seq_info{0, 0, 0});
        rc = parse_info(args.infoPath, &info, args.infoLen, args.seqLen);
        if (rc != SUCCESS) return rc;
    }
    if (args.airr) rc = parse_airr_input(args.seqPath, &seqs, &info, args.seqLen, overlap);
    else rc = parse_input(args.seqPath, &seqs, &info, args.seqLen, overlap);
    if (rc != SUCCESS) return rc;

    const double t_parse = ms_since(t_main);
    if (args.verbose) print_args(args);
    Sink sink;
    if (args.outputPath) {
        sink.out = fopen(args.outputPath, "w");
        if (!sink.out) return print_err("output file opening failed");
    }
    xtn_args xa{args.distance, args.measure, args.verbose, args.infoLen};
    init.join();
    int r = ctx_rc;
    if (r != XTN_SUCCESS) return print_err(init_err.c_str());
    const double t_init = ms_since(t_main);
    double t_search = t_init;
    xtn_stats st{};
    if (r == XTN_SUCCESS) {
        r = xtn_context_perform(ctx, &xa, seqs.chars.data(), seqs.offsets.data(), seqs.size(),
                                overlap ? info.data() : nullptr, overlap ? overlap_handler : nn_handler, &sink);
        t_search = ms_since(t_main);
        xtn_context_stats(ctx, &st);
    }
    std::string err = r != XTN_SUCCESS ? xtn_last_error() : "";
    xtn_context_destroy(ctx);
    ctx = nullptr;
    if (sink.out && fclose(sink.out) != 0) sink.failed = true;
    if (r != XTN_SUCCESS) return print_err(err.c_str());
    if (sink.failed) return print_err("output file writing failed");
    if (args.verbose) {
        // host-time breakdown of this process from main() on (the exec and library loading
        // before main() and the exit after it are outside): input parse, CUDA start-up (on
        // its own thread during the parse) and what was left of it after the parse, search
        // with output delivery (the device time of the search itself), release
        const double t_end = ms_since(t_main);
        printf("xtn_b200 stage parse %.3f\n", t_parse);
        printf("xtn_b200 stage cuda_init %.3f\n", t_init_done);  // from main(), beside the parse
        printf("xtn_b200 stage wait_for_cuda_init %.3f\n", t_init - t_parse);
        printf("xtn_b200 stage search_and_output %.3f\n", t_search - t_init);
        printf("xtn_b200 stage device_search %.3f\n", st.ms_total);
        printf("xtn_b200 stage release %.3f\n", t_end - t_search);
        printf("total output length: %'lu\n", (unsigned long)sink.total);
    }
    return SUCCESS;
}
