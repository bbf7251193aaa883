// text_input.cpp -- libsvm text files ("label idx:val idx:val ...") into an
// svm_problem, parsed by all host threads at once.
//
// Acceptance rules are those of the reference's read_problem
// (svm-train/svm-train.c:288-389), which tokenises each line with strtok:
//   * the label is the first token delimited by space, tab or newline and
//     must be a whole strtod number; a line without one (empty or blank) is
//     malformed;
//   * each feature is an index token running from the current position to the
//     next ':' (leading ':' skipped) and a value token delimited by space or
//     tab; the loop ends when no value token is left, so trailing text
//     without a ':' is ignored;
//   * the index must be a whole base-10 strtol number that fits, strictly
//     greater than the previous index of the line (the first may be 0); the
//     value a strtod number without range error followed by nothing or by
//     whitespace.
// The first malformed line (1-based) is reported, as the reference reports
// it.  Numbers are converted with strtod/strtol, so values are bit-identical
// to the reference's.
//
// Parallel layout: the file is mapped (or read whole), cut into one byte
// range per thread at line starts; each thread parses its lines into its own buffers,
// and the buffers are concatenated into one node array (rows terminated by
// index -1, as svm_node lists are).
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <chrono>

#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "engine.hpp"
#include "svm.h"
#include "svm_b200.h"

namespace svmb {
namespace {

struct Part {
    std::vector<double> y;
    std::vector<svm_node> nodes;     // rows terminated by index -1
    long long lines = 0;
    long long bad_line = 0;          // first malformed line within the part (1-based), 0 if none
    int max_index = 0;
};

inline bool is_blank(char c) { return c == ' ' || c == '\t'; }

// A number token as a NUL-terminated string (tokens are short; the copy keeps
// strtod/strtol from seeing past the token).
struct Tok {
    char small[128];
    std::string big;
    const char *set(const char *a, const char *b)
    {
        const size_t n = (size_t)(b - a);
        if (n < sizeof small) {
            memcpy(small, a, n);
            small[n] = 0;
            return small;
        }
        big.assign(a, n);
        return big.c_str();
    }
};

// Parse one line [a, e) (e is past the line's '\n', or the end of the file).
// Returns false if the line is malformed.
bool parse_line(const char *a, const char *e, Part &P, Tok &tok)
{
    // label: first token delimited by " \t\n"
    const char *p = a;
    while (p < e && (is_blank(*p) || *p == '\n')) ++p;
    if (p == e) return false;
    const char *q = p;
    while (q < e && !is_blank(*q) && *q != '\n') ++q;
    {
        const char *s = tok.set(p, q);
        char *end;
        const double v = strtod(s, &end);
        if (end == s || *end != '\0') return false;
        P.y.push_back(v);
    }
    // the delimiter after the label is consumed (strtok writes its NUL there)
    p = q < e ? q + 1 : e;
    int last = -1;
    while (true) {
        // index token: skip ':' then run to the next ':' (or the end)
        while (p < e && *p == ':') ++p;
        if (p == e) break;
        const char *ib = p;
        while (p < e && *p != ':') ++p;
        const char *ie = p;
        if (p < e) ++p;              // the ':' delimiter
        // value token: skip blanks, run to the next blank (or the end)
        while (p < e && is_blank(*p)) ++p;
        if (p == e) break;           // no value token: the loop ends
        const char *vb = p;
        while (p < e && !is_blank(*p)) ++p;
        const char *ve = p;
        if (p < e) ++p;              // the blank delimiter
        svm_node nd;
        {
            const char *s = tok.set(ib, ie);
            char *end;
            errno = 0;
            const long idx = strtol(s, &end, 10);
            nd.index = (int)idx;
            if (end == s || errno != 0 || *end != '\0' || nd.index <= last) return false;
            last = nd.index;
        }
        {
            const char *s = tok.set(vb, ve);
            char *end;
            errno = 0;
            nd.value = strtod(s, &end);
            if (end == s || errno != 0 || (*end != '\0' && !isspace((unsigned char)*end))) return false;
        }
        P.nodes.push_back(nd);
    }
    if (last > P.max_index) P.max_index = last;
    svm_node term;
    term.index = -1;
    term.value = 0;
    P.nodes.push_back(term);
    return true;
}

void parse_range(const char *a, const char *e, Part &P)
{
    Tok tok;
    while (a < e) {
        const char *nl = (const char *)memchr(a, '\n', (size_t)(e - a));
        const char *le = nl ? nl + 1 : e;
        ++P.lines;
        if (!P.bad_line && !parse_line(a, le, P, tok)) P.bad_line = P.lines;
        if (P.bad_line) {
            // the rest of the part only needs its line count
            for (const char *c = le; c < e;) {
                const char *n2 = (const char *)memchr(c, '\n', (size_t)(e - c));
                ++P.lines;
                c = n2 ? n2 + 1 : e;
            }
            return;
        }
        a = le;
    }
}

}  // namespace
}  // namespace svmb

extern "C" {

int svmb_read_problem(const char *path, struct svm_problem *prob, struct svm_node **x_space, int *max_index,
                      long long *bad_line)
{
    using namespace svmb;
    if (!path || !prob || !x_space) {
        set_error("invalid arguments");
        return -1;
    }
    if (bad_line) *bad_line = 0;
    const auto c0 = std::chrono::steady_clock::now();
    auto since = [](std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
    };
    // A regular file is mapped: its pages are faulted in by the threads that
    // parse them, in parallel.  Anything else (a pipe, say) is read whole.
    const char *base = nullptr;
    size_t size = 0;
    std::vector<char> buf;
    void *map = MAP_FAILED;
    {
        const int fd = open(path, O_RDONLY);
        if (fd < 0) {
            set_error(std::string("can't open input file ") + path);
            return -1;
        }
        struct stat st;
        if (fstat(fd, &st) == 0 && S_ISREG(st.st_mode) && st.st_size > 0) {
            size = (size_t)st.st_size;
            map = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
            if (map != MAP_FAILED) base = (const char *)map;
        }
        if (!base) {
            size = 0;
            buf.resize(1 << 20);
            while (true) {
                const ssize_t got = read(fd, buf.data() + size, buf.size() - size);
                if (got < 0) {
                    close(fd);
                    set_error(std::string("error reading ") + path);
                    return -1;
                }
                if (got == 0) break;
                size += (size_t)got;
                if (size == buf.size()) buf.resize(buf.size() * 2);
            }
            base = buf.data();
        }
        close(fd);
    }
    struct Unmap {
        void *p;
        size_t n;
        ~Unmap() { if (p != MAP_FAILED) munmap(p, n); }
    } unmap{map, size};

    // byte ranges at line starts, one per thread (small files: one range)
    const int threads = size < (1u << 20) ? 1 : std::max(1, omp_get_max_threads());
    std::vector<size_t> cut(threads + 1, size);
    cut[0] = 0;
    for (int t = 1; t < threads; t++) {
        size_t c = std::max(cut[t - 1], size * (size_t)t / (size_t)threads);
        if (c > 0 && c < size && base[c - 1] != '\n') {
            const char *nl = (const char *)memchr(base + c, '\n', size - c);
            c = nl ? (size_t)(nl - base) + 1 : size;
        }
        cut[t] = c;
    }
    const double t_read = since(c0);
    std::vector<Part> parts(threads);
#pragma omp parallel for schedule(static, 1) num_threads(threads)
    for (int t = 0; t < threads; t++) parse_range(base + cut[t], base + cut[t + 1], parts[t]);
    const double t_parse = since(c0) - t_read;
    long long line0 = 0;
    for (int t = 0; t < threads; t++) {
        if (parts[t].bad_line) {
            if (bad_line) *bad_line = line0 + parts[t].bad_line;
            set_error("Wrong input format at line " + std::to_string(line0 + parts[t].bad_line));
            return -2;
        }
        line0 += parts[t].lines;
    }
    // concatenate
    size_t rows = 0, nodes = 0;
    int maxi = 0;
    std::vector<size_t> row0(threads), node0(threads);
    for (int t = 0; t < threads; t++) {
        row0[t] = rows;
        node0[t] = nodes;
        rows += parts[t].y.size();
        nodes += parts[t].nodes.size();
        maxi = std::max(maxi, parts[t].max_index);
    }
    if (rows > (size_t)0x7fffffff) {
        set_error("too many rows");
        return -1;
    }
    double *y = (double *)malloc(sizeof(double) * std::max<size_t>(rows, 1));
    svm_node **x = (svm_node **)malloc(sizeof(svm_node *) * std::max<size_t>(rows, 1));
    svm_node *space = (svm_node *)malloc(sizeof(svm_node) * std::max<size_t>(nodes, 1));
    if (!y || !x || !space) {
        free(y);
        free(x);
        free(space);
        set_error("out of host memory");
        return -1;
    }
#pragma omp parallel for schedule(static, 1) num_threads(threads)
    for (int t = 0; t < threads; t++) {
        const Part &P = parts[t];
        memcpy(y + row0[t], P.y.data(), sizeof(double) * P.y.size());
        memcpy(space + node0[t], P.nodes.data(), sizeof(svm_node) * P.nodes.size());
        size_t r = row0[t], k = node0[t];
        const size_t kend = node0[t] + P.nodes.size();
        while (k < kend) {
            x[r++] = space + k;
            while (space[k].index != -1) ++k;
            ++k;
        }
    }
    prob->l = (int)rows;
    prob->y = y;
    prob->x = x;
    *x_space = space;
    if (getenv("SVMB_TRACE") && *getenv("SVMB_TRACE") == '1')
        fprintf(stderr, "[svmb] read_problem %s threads=%d read=%.1fms parse=%.1fms assemble=%.1fms\n", path, threads,
                t_read, t_parse, since(c0) - t_read - t_parse);
    if (max_index) *max_index = maxi;
    return 0;
}

void svmb_free_problem(struct svm_problem *prob, struct svm_node *x_space)
{
    if (prob) {
        free(prob->y);
        free(prob->x);
        prob->y = NULL;
        prob->x = NULL;
        prob->l = 0;
    }
    free(x_space);
}

}  // extern "C"
