// The SDPA sparse-format reader behind brisk_solve_file and bgpu_sdpa_read: the reference's
// read_sdpa (problem.c:426-575) with its tokenizers next_num and line_num (problem.c:58-91).
//
// The file is read into memory once.  Separators ",{}()=" become blanks and Fortran exponents
// ("1.5D+03") become 'e', as the reference's first pass does; here both run on all host threads
// (the exponent rule looks only at character classes that those rewrites never change, so the
// positions are found first and written after).  The header (m, nblk, the block sizes, c) is read
// serially with the reference's rules.  The entries, the bulk of every large file, are parsed in
// parallel: the data section is cut at blanks into one piece per thread, each piece's words are
// counted, then converted into one array at the piece's offset, and the numbers are grouped five
// by five across the pieces; the checks of each entry (integer indices, finite value, ranges) run
// in parallel and the first failing entry in file order is the one reported.  That form needs every
// word of the data section to be one plain number that starts with a digit, a sign or a point:
// any other word (text after the last entry, a number glued to text, "inf") sends the data section
// to the serial reader, a restatement of the reference's loop token by token.
//
// Numbers: std::from_chars is correctly rounded, so it gives strtod's double bit for bit (as the
// reference's Clinger fast path does, problem.c:29-55, where it applies); strtod takes the forms
// from_chars does not (a leading '+', hexadecimal, results out of the normal range).
#include "solver.h"

#include <algorithm>
#include <cfloat>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>
#include <thread>
#include <vector>

namespace bsolve {
namespace {

constexpr int kReadMaxN = 46340;   // the largest SDP block read (problem.c:326, g_read_maxn)

inline bool blank(unsigned char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }   // C isspace
inline bool digit(unsigned char c) { return c >= '0' && c <= '9'; }

// strtod's value of the word [p, e) (*e a blank or the terminating NUL); false when strtod does not
// read the whole word as one number.
inline bool word_number(const char *p, const char *e, double &v) {
    const auto r = std::from_chars(p, e, v);
    if (r.ec == std::errc() && r.ptr == e && std::isfinite(v) && (v == 0 || std::fabs(v) >= DBL_MIN)) return true;
    char *end;
    v = std::strtod(p, &end);
    return end == e;
}

// next_num (problem.c:58-73): the next number; a word that is not one is skipped and counted, a
// number glued to text is taken and the text counted.  False at the end of the text.
bool next_num(char *&p, double &out, long &skipped) {
    for (;;) {
        while (*p && blank(*p)) p++;
        if (!*p) return false;
        char *w = p;
        while (*w && !blank(*w)) w++;
        double v;
        if (word_number(p, w, v)) {
            out = v;
            p = w;
            return true;
        }
        char *e;
        v = std::strtod(p, &e);
        if (e != p) {
            out = v;
            p = e;
            skipped++;
            return true;
        }
        p = w;
        skipped++;
    }
}

// line_num (problem.c:75-91): the first number on the next line that does not start with '"' or
// '*'; the rest of that line is passed over (its newline becomes a blank, as there).
bool line_num(char *&p, double &out, long &skipped) {
    while (*p) {
        char *eol = std::strchr(p, '\n');
        char *next = eol ? eol + 1 : p + std::strlen(p);
        if (eol) *eol = '\0';
        char *q = p;
        while (*q && blank(*q)) q++;
        bool ok = false;
        if (*q && *q != '"' && *q != '*') ok = next_num(q, out, skipped);
        if (eol) *eol = ' ';
        p = next;
        if (ok) return true;
    }
    return false;
}

int host_threads(size_t bytes) {
    unsigned t = std::thread::hardware_concurrency();
    t = std::max(1u, std::min(t, 32u));
    const size_t per = (size_t)4 << 20;   // below 4 MB a thread is not worth starting
    return (int)std::max<size_t>(1, std::min<size_t>(t, bytes / per));
}

template <typename F>
void on_threads(int nt, F f) {
    if (nt == 1) {
        f(0);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++) th.emplace_back(f, t);
    for (auto &x : th) x.join();
}

char *cut(char *lo, char *end, int t, int nt) {   // piece t's start, at a blank
    if (t == 0) return lo;
    if (t == nt) return end;
    char *x = lo + (size_t)(end - lo) * t / nt;
    while (x < end && !blank(*x)) x++;
    return x;
}

// Separators and Fortran exponents (problem.c:436-444) on the piece [lo, hi) of a text of len
// characters: `before` is the character at lo - 1, after0/after1 those at hi and hi + 1 (0 where
// the text has none), so that a piece is rewritten without reading another thread's piece.  The
// exponent rule sees the classes "digit or point" and "sign" only, which neither rewrite changes,
// so the order of the rewrites inside the piece does not matter.
// Returns whether the piece holds a NUL (the text then ends there, as a C string).
bool rewrite_piece(char *buf, size_t lo, size_t hi, size_t len, char before, char after0, char after1) {
    auto at = [&](size_t i) -> unsigned char {
        if (i < lo) return (unsigned char)before;
        if (i < hi) return (unsigned char)buf[i];
        return (unsigned char)(i == hi ? after0 : after1);
    };
    bool nul = false;
    for (size_t i = lo; i < hi; i++) {
        const char ch = buf[i];
        nul |= ch == '\0';
        if (ch == ',' || ch == '{' || ch == '}' || ch == '(' || ch == ')' || ch == '=') {
            buf[i] = ' ';
        } else if ((ch == 'D' || ch == 'd') && i > 0 && i + 1 < len) {
            const unsigned char a = at(i - 1), b = at(i + 1);
            if ((digit(a) || a == '.') &&
                (digit(b) || ((b == '+' || b == '-') && i + 2 < len && digit(at(i + 2)))))
                buf[i] = 'e';
        }
    }
    return nul;
}

// The whole file into buf (len characters and a NUL), read and rewritten by one thread per piece
// (pread of the piece and of its three neighbouring characters).  False on a read error or a file
// that changed size while read; *nul: the text holds a NUL.
bool read_rewrite(int fd, size_t len, char *buf, bool *nul) {
    const int nt = host_threads(len);
    std::vector<char> ok(nt, 1), has_nul(nt, 0);
    auto rd = [&](char *dst, size_t n, size_t off) {
        while (n) {
            const ssize_t got = pread(fd, dst, n, (off_t)off);
            if (got <= 0) return false;
            dst += got;
            n -= (size_t)got;
            off += (size_t)got;
        }
        return true;
    };
    on_threads(nt, [&](int t) {
        const size_t lo = len * t / nt, hi = len * (t + 1) / nt;
        char nb[3] = {0, 0, 0};
        const size_t tail = std::min<size_t>(2, len - hi);
        if (!rd(buf + lo, hi - lo, lo) || (lo > 0 && !rd(nb, 1, lo - 1)) || (tail && !rd(nb + 1, tail, hi))) {
            ok[t] = 0;
            return;
        }
        has_nul[t] = rewrite_piece(buf, lo, hi, len, nb[0], nb[1], nb[2]);
    });
    buf[len] = '\0';
    *nul = false;
    for (int t = 0; t < nt; t++) {
        if (!ok[t]) return false;
        *nul |= has_nul[t] != 0;
    }
    return true;
}

// Comment lines from p on: lines whose first character after ' ', '\t', '\r' is '"' or '*' are
// blanked (problem.c:454-466).  A line belongs to the thread whose piece holds its start; the
// starts are found (read only) before any line is written.
void blank_comments(char *p, char *end) {
    const size_t len = (size_t)(end - p);
    const int nt = host_threads(len);
    std::vector<char *> start(nt + 1, end);
    start[0] = p;
    on_threads(nt, [&](int t) {
        if (t == 0) return;
        char *x = p + len * t / nt;   // the first line start at or after the piece's nominal start
        while (x < end && !(x == p || x[-1] == '\n')) x++;
        start[t] = x;
    });
    on_threads(nt, [&](int t) {
        char *q = start[t];
        const char *hi = t + 1 < nt ? start[t + 1] : end;
        while (q < hi) {
            char *eol = (char *)std::memchr(q, '\n', (size_t)(end - q));
            char *e = eol ? eol : end;
            char *s = q;
            while (s < e && (*s == ' ' || *s == '\t' || *s == '\r')) s++;
            if (s < e && (*s == '"' || *s == '*'))
                for (char *x = q; x < e; x++) *x = ' ';
            if (!eol) break;
            q = eol + 1;
        }
    });
}

enum EntryFault { kOk = 0, kNonInteger, kNonFinite, kBadEntry, kLpOffDiagonal };

// The checks of one entry in the reference's order (problem.c:528-548); kOk with keep = false for
// a zero value.
EntryFault check_entry(const double *e, int m, int nblk, const int *bs, bool &keep) {
    keep = false;
    for (int q = 0; q < 4; q++)
        if (e[q] != std::floor(e[q]) || std::fabs(e[q]) > 2e9) return kNonInteger;
    if (!std::isfinite(e[4])) return kNonFinite;
    if (e[4] == 0.0) return kOk;
    const int mat = (int)e[0], bk = (int)e[1] - 1, i = (int)e[2] - 1, j = (int)e[3] - 1;
    if (mat < 0 || mat > m || bk < 0 || bk >= nblk) return kBadEntry;
    const int n = std::abs(bs[bk]);
    if (i < 0 || j < 0 || i >= n || j >= n) return kBadEntry;
    if (bs[bk] < 0 && i != j) return kLpOffDiagonal;
    keep = true;
    return kOk;
}

std::string fault_text(EntryFault f, const double *e) {
    char s[256];
    switch (f) {
    case kNonInteger:
        std::snprintf(s, sizeof s, "non-integer index in entry %g %g %g %g %g", e[0], e[1], e[2], e[3], e[4]);
        break;
    case kNonFinite:
        std::snprintf(s, sizeof s, "non-finite value in entry %g %g %g %g", e[0], e[1], e[2], e[3]);
        break;
    case kBadEntry:
        std::snprintf(s, sizeof s, "bad entry %d %d %d %d", (int)e[0], (int)e[1], (int)e[2], (int)e[3]);
        break;
    default:
        std::snprintf(s, sizeof s, "off-diagonal entry in LP block");
        break;
    }
    return s;
}

void push(InputData &in, const double *e) {
    in.mat.push_back((int)e[0]);
    in.blk.push_back((int)e[1]);
    in.i.push_back((int)e[2]);
    in.j.push_back((int)e[3]);
    in.v.push_back(e[4]);
}

// The data section token by token (problem.c:497-566), for text the parallel form does not take.
int entries_serial(char *p, const char *path, InputData &in, std::string &err) {
    long skipped = 0;
    double e[5];
    for (;;) {
        char *q = p;
        while (*q && blank(*q)) q++;
        if (*q && !(digit(*q) || *q == '-' || *q == '+' || *q == '.')) {
            // at an entry boundary, a word that starts no number: the end of the data when no later
            // line holds five numbers (text after the last entry), else the error below
            bool more = false;
            long nl = 0;
            for (char *r = q; *r && !more;) {
                char *eol = std::strchr(r, '\n');
                const size_t len = eol ? (size_t)(eol - r) : std::strlen(r);
                nl++;
                char *t = r;
                int nnum = 0;
                while (t < r + len) {
                    while (t < r + len && blank(*t)) t++;
                    if (t >= r + len) break;
                    char *e2;
                    (void)std::strtod(t, &e2);
                    if (e2 == t) break;
                    nnum++;
                    t = e2;
                }
                if (nnum >= 5) more = true;
                r = eol ? eol + 1 : r + len;
            }
            if (!more) {
                log_printf(1, "brisk: note: %ld line(s) of text after the last entry of %s ignored\n", nl, path);
                break;
            }
        }
        int got = 0;
        for (; got < 5; got++)
            if (!next_num(p, e[got], skipped)) break;
        if (got < 5) {
            if (got > 0) log_printf(1, "brisk: warning: incomplete last entry (%d of 5 numbers) ignored\n", got);
            break;
        }
        bool keep;
        const EntryFault f = check_entry(e, in.m, in.nblk, in.bs.data(), keep);
        if (f != kOk) {
            err = fault_text(f, e);
            return 2;
        }
        if (keep) push(in, e);
    }
    if (skipped) {
        err = std::to_string(skipped) + " non-numeric token(s) in the data section of " + path +
              " (every entry is \"matrix block i j value\", numbers only)";
        return 2;
    }
    return 0;
}

// The data section on all host threads; returns -1 (nothing changed in `in`) when a word is not a
// plain number, so that the serial reader takes the section.  Each piece's numbers go to its own
// array (a piece of B characters holds at most B/2 + 1 words); an entry belongs to the piece that
// holds its first number and may take the rest from the pieces after it.
int entries_parallel(char *p, char *end, InputData &in, std::string &err) {
    const int nt = host_threads((size_t)(end - p));
    std::vector<char *> bound(nt + 1);
    for (int t = 0; t <= nt; t++) bound[t] = cut(p, end, t, nt);
    for (int t = 1; t <= nt; t++) bound[t] = std::max(bound[t], bound[t - 1]);
    std::vector<std::vector<double, NoInitAlloc<double>>> num(nt);
    std::vector<size_t> words(nt + 1, 0);
    std::vector<char> plain(nt, 1);
    on_threads(nt, [&](int t) {
        num[t].resize((size_t)(bound[t + 1] - bound[t]) / 2 + 1);
        double *out = num[t].data();
        const char *x = bound[t], *hi = bound[t + 1];
        for (;;) {
            while (x < hi && blank(*x)) x++;
            if (x >= hi) break;
            const char *w = x;
            while (w < hi && !blank(*w)) w++;
            const unsigned char c0 = *x;
            if (!(digit(c0) || c0 == '-' || c0 == '+' || c0 == '.') || !word_number(x, w, *out)) {
                plain[t] = 0;
                return;
            }
            out++;
            x = w;
        }
        words[t + 1] = (size_t)(out - num[t].data());
    });
    for (int t = 0; t < nt; t++)
        if (!plain[t]) return -1;
    for (int t = 0; t < nt; t++) words[t + 1] += words[t];
    const size_t N = words[nt], nent = N / 5;
    if (N % 5) log_printf(1, "brisk: warning: incomplete last entry (%d of 5 numbers) ignored\n", (int)(N % 5));
    // entries [e0[t], e0[t + 1]) start in piece t
    std::vector<size_t> e0(nt + 1);
    for (int t = 0; t <= nt; t++) e0[t] = std::min(nent, (words[t] + 4) / 5);
    auto fetch = [&](int t, size_t k, double *e) {   // entry k's numbers, from piece t on
        size_t g = 5 * k;
        for (int q = 0; q < 5; q++, g++) {
            while (g >= words[t + 1]) t++;
            e[q] = num[t][g - words[t]];
        }
    };
    std::vector<size_t> kept(nt + 1, 0), first_bad(nt, nent);
    std::vector<EntryFault> fault(nt, kOk);
    const int *bs = in.bs.data();
    on_threads(nt, [&](int t) {
        size_t c = 0;
        double e[5];
        for (size_t k = e0[t]; k < e0[t + 1]; k++) {
            fetch(t, k, e);
            bool keep;
            const EntryFault f = check_entry(e, in.m, in.nblk, bs, keep);
            if (f != kOk) {
                first_bad[t] = k;
                fault[t] = f;
                return;
            }
            c += keep;
        }
        kept[t + 1] = c;
    });
    for (int t = 0; t < nt; t++)
        if (fault[t] != kOk) {   // the earliest piece with a fault holds the first one in file order
            double e[5];
            fetch(t, first_bad[t], e);
            err = fault_text(fault[t], e);
            return 2;
        }
    for (int t = 0; t < nt; t++) kept[t + 1] += kept[t];
    const size_t nk = kept[nt];
    in.mat.resize(nk);
    in.blk.resize(nk);
    in.i.resize(nk);
    in.j.resize(nk);
    in.v.resize(nk);
    on_threads(nt, [&](int t) {
        size_t o = kept[t];
        double e[5];
        for (size_t k = e0[t]; k < e0[t + 1]; k++) {
            fetch(t, k, e);
            if (e[4] == 0.0) continue;
            in.mat[o] = (int)e[0];
            in.blk[o] = (int)e[1];
            in.i[o] = (int)e[2];
            in.j[o] = (int)e[3];
            in.v[o] = e[4];
            o++;
        }
    });
    return 0;
}

}  // namespace

// Fills `in` in the SDPA numbering as brisk_solve_data takes it (1-based, F0 as mat 0, zero values
// left out, an entry of the lower triangle kept as given); 0, or 2 with err set.
int read_sdpa_file(const char *path, InputData &in, std::string &err) {
    in = InputData();
    const std::string malformed = std::string("malformed SDPA file ") + path;
    const int fd = open(path, O_RDONLY);
    if (fd < 0) {
        err = std::string("cannot open ") + path;
        return 2;
    }
    struct stat st;
    if (fstat(fd, &st) != 0 || S_ISDIR(st.st_mode)) {
        close(fd);
        err = S_ISDIR(st.st_mode) ? std::string(path) + " is a directory, not an SDPA file" : std::string("cannot read ") + path;
        return 2;
    }
    std::vector<char, NoInitAlloc<char>> buf;
    bool read_ok = false, nul = false;
    if (S_ISREG(st.st_mode)) {
        buf.resize((size_t)st.st_size + 1);
        read_ok = read_rewrite(fd, (size_t)st.st_size, buf.data(), &nul);
    } else {   // a pipe or a device: read to the end, then rewrite on this thread
        size_t cap = 1 << 20, len = 0;
        buf.resize(cap + 1);
        for (;;) {
            if (len == cap) {
                cap *= 2;
                buf.resize(cap + 1);
            }
            const ssize_t got = read(fd, buf.data() + len, cap - len);
            if (got < 0) break;
            if (got == 0) {
                read_ok = true;
                break;
            }
            len += (size_t)got;
        }
        buf.resize(len + 1);
        buf[len] = '\0';
        nul = rewrite_piece(buf.data(), 0, len, len, 0, 0, 0);
    }
    close(fd);
    if (!read_ok) {
        err = std::string("cannot read ") + path;
        return 2;
    }
    const size_t len = buf.size() - 1;
    char *p = buf.data(), *end = buf.data() + len;
    if (nul) end = p + std::strlen(p);   // the text ends at a NUL, as a C string
    long skipped = 0;
    double v;
    if (!line_num(p, v, skipped)) {
        err = malformed;
        return 2;
    }
    const double vm = v;
    if (!line_num(p, v, skipped)) {
        err = malformed;
        return 2;
    }
    blank_comments(p, end);
    // (the ranges keep the casts defined; m and nblk cannot exceed the numbers left in the text)
    const size_t left = (size_t)(end - p);
    if (!(vm > -1 && vm < 100000001.0) || !(v >= 1 && v < 2147483648.0) || v != std::floor(v) ||
        (size_t)v > left || (size_t)vm > left) {
        err = malformed;
        return 2;
    }
    const int m = (int)vm, nblk = (int)v;
    in.m = m;
    in.nblk = nblk;
    in.bs.resize(nblk);
    for (int k = 0; k < nblk; k++) {
        if (!next_num(p, v, skipped)) {
            err = malformed;
            return 2;
        }
        if (!(std::fabs(v) >= 1 && std::fabs(v) <= 2e9) || v != std::floor(v)) {
            char s[96];
            std::snprintf(s, sizeof s, "invalid size %g of block %d", v, k + 1);
            err = s;
            return 2;
        }
        in.bs[k] = (int)v;
    }
    in.c.resize(m);
    for (int i = 0; i < m; i++) {
        if (!next_num(p, v, skipped) || !std::isfinite(v)) {
            err = malformed;
            return 2;
        }
        in.c[i] = v;
    }
    int rc = entries_parallel(p, end, in, err);
    if (rc < 0) rc = entries_serial(p, path, in, err);
    if (rc) return rc;
    for (int k = 0; k < nblk; k++)
        if (in.bs[k] > kReadMaxN) {
            err = "SDP block " + std::to_string(k + 1) + " of size " + std::to_string(in.bs[k]) +
                  " exceeds the supported maximum (46340)";
            return 2;
        }
    return 0;
}

}  // namespace bsolve
