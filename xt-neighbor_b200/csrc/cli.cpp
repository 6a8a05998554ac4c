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
#include <chrono>
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

// S/src/cli.cu:101-147
int parse_input(const char* path, SeqStore* seqs, std::vector<xtn_seq_info>* info, int len, bool doubleCol) {
    FILE* f = fopen(path, "r");
    if (!f) return print_err("input file reading failed");
    PieceReader rd(f, 500);
    int lineNumber = 1, count = 0;
    rd.next();  // header
    while (rd.next()) {
        lineNumber++;
        char* line = rd.line();
        if (blank_line(line)) continue;
        int r = seqs->append(line);
        if (r != SUCCESS) {
            fclose(f);
            return print_err_line("input parsing error", lineNumber);
        }
        if (doubleCol) {
            char* c = strchr(line, ',');
            if (!c) {
                fclose(f);
                return print_err_line("input parsing error (comma expected)", lineNumber);
            }
            int v;
            if (!parse_int_field(c + 1, &v)) {
                fclose(f);
                return print_err_line("input parsing error (invalid number)", lineNumber);
            }
            if (count < (int)info->size()) (*info)[count].frequency = v;
        }
        count++;
    }
    fclose(f);
    if (count != len) return print_err("input length doesn't match with the actual");
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
    // the library context: device selection, CUDA context creation, stream and pinned scalars
    xtn_context* ctx = nullptr;
    int r = xtn_context_create(0, &ctx);
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
    if (sink.out && fclose(sink.out) != 0) sink.failed = true;
    if (r != XTN_SUCCESS) return print_err(err.c_str());
    if (sink.failed) return print_err("output file writing failed");
    if (args.verbose) {
        // host-time breakdown of this process from main() on (the exec and library loading
        // before main() and the exit after it are outside): input parse, CUDA start-up,
        // search with output delivery (the device time of the search itself), release
        const double t_end = ms_since(t_main);
        printf("xtn_b200 stage parse %.3f\n", t_parse);
        printf("xtn_b200 stage cuda_init %.3f\n", t_init - t_parse);
        printf("xtn_b200 stage search_and_output %.3f\n", t_search - t_init);
        printf("xtn_b200 stage device_search %.3f\n", st.ms_total);
        printf("xtn_b200 stage release %.3f\n", t_end - t_search);
        printf("total output length: %'lu\n", (unsigned long)sink.total);
    }
    return SUCCESS;
}
