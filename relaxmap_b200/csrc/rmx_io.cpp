// Input parsing and output writing with the reference's exact rules.
//
// Both reference loaders read lines with getline and split them with
// `istringstream >> string` into one string variable `buf` that lives across
// lines. A read that finds no token leaves `buf` unchanged, so a blank line in
// an edge list re-reads the previous line's last token. After any processed
// line `buf` holds that line's third token or "" (it is cleared before the
// weight is read), so the state entering a line depends only on the previous
// processed line: the parser below reproduces it, also across the chunk
// boundaries of the multi-threaded edge-list parse.
#include "rmx_io.hpp"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <map>
#include <mutex>
#include <thread>
#include <utility>

namespace rmx {

namespace {

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

struct Tok {
    const char *b = nullptr, *e = nullptr;
    bool empty() const { return b == e; }
    std::string str() const { return std::string(b, e); }
};

// One line as an istringstream: successive >> reads until the first failure.
struct LineStream {
    const char *p, *end;
    bool failed = false;
    LineStream(const char *b, const char *e) : p(b), end(e) {}
    // istringstream >> buf: on failure buf is left as it was
    void read(Tok &buf) {
        if (failed) return;
        while (p < end && is_ws(*p)) p++;
        if (p == end) {
            failed = true;
            return;
        }
        const char *s = p;
        while (p < end && !is_ws(*p)) p++;
        buf.b = s;
        buf.e = p;
    }
};

// C atol / atoi on a token (the token has no leading whitespace).
long long c_atol(const Tok &t) {
    const char *p = t.b;
    bool neg = false;
    if (p < t.e && (*p == '+' || *p == '-')) neg = *p++ == '-';
    unsigned long long v = 0;
    while (p < t.e && *p >= '0' && *p <= '9') v = v * 10 + (unsigned)(*p++ - '0');
    return (long long)(neg ? 0ull - v : v);  // negated unsigned: -2^63 has no signed negation
}

// C atof (strtod) on a token. A token that is a plain decimal
// [+-]digits[.digits] whose digits form an integer m < 2^53 with at most 22 of
// them after the point takes Clinger's fast path (W. D. Clinger, "How to read
// floating point numbers accurately", PLDI 1990): m and 10^k are then exact
// doubles, so the one IEEE division m / 10^k is the correctly rounded value of
// the decimal, which is what glibc's strtod returns. Any other token (an
// exponent, inf/nan, hex, more digits, trailing characters) goes to strtod.
double c_atof(const Tok &t) {
    static const double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                      1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};
    {
        const char *p = t.b;
        bool neg = false;
        if (p < t.e && (*p == '+' || *p == '-')) neg = *p++ == '-';
        uint64_t m = 0;
        int digits = 0, frac = 0;
        bool fast = true, point = false;
        for (; p < t.e && fast; p++) {
            const char c = *p;
            if (c >= '0' && c <= '9') {
                m = m * 10 + (uint64_t)(c - '0');
                digits++;
                if (point) frac++;
                fast = m < (uint64_t(1) << 53) && frac <= 22;
            } else if (c == '.' && !point) {
                point = true;
            } else {
                fast = false;
            }
        }
        if (fast && digits > 0) {
            const double v = (double)m / kPow10[frac];
            return neg ? -v : v;
        }
    }
    char buf[96];
    size_t n = (size_t)(t.e - t.b);
    if (n < sizeof buf) {
        memcpy(buf, t.b, n);
        buf[n] = 0;
        return strtod(buf, nullptr);
    }
    std::string s(t.b, t.e);
    return strtod(s.c_str(), nullptr);
}

// The bytes of a file: a read-only mapping of a regular file (the parser
// threads fault its pages in themselves), else what reads from the stream
// returned (pipes, devices). As with any mapped read, a file that another
// process truncates while it is parsed raises SIGBUS.
class FileBytes {
  public:
    FileBytes() = default;
    FileBytes(const FileBytes &) = delete;
    FileBytes &operator=(const FileBytes &) = delete;
    FileBytes(FileBytes &&o) noexcept { *this = std::move(o); }
    FileBytes &operator=(FileBytes &&o) noexcept {
        if (this != &o) {
            release();
            map_ = o.map_;
            n_ = o.n_;
            buf_ = std::move(o.buf_);
            o.map_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    ~FileBytes() { release(); }
    const char *data() const { return map_ ? static_cast<const char *>(map_) : buf_.data(); }
    size_t size() const { return map_ ? n_ : buf_.size(); }
    char operator[](size_t i) const { return data()[i]; }
    void release() {
        if (map_) munmap(map_, n_);
        map_ = nullptr;
        n_ = 0;
        std::vector<char>().swap(buf_);
    }
    static FileBytes read(const std::string &path);

  private:
    void *map_ = nullptr;
    size_t n_ = 0;
    std::vector<char> buf_;
};

FileBytes FileBytes::read(const std::string &path) {
    FileBytes out;
    const int fd = open(path.c_str(), O_RDONLY);
    if (fd < 0) throw IoError("cannot open " + path + ": " + strerror(errno));
    struct stat st;
    if (fstat(fd, &st) == 0 && S_ISREG(st.st_mode) && st.st_size > 0) {
        void *m = mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
        if (m != MAP_FAILED) {
            madvise(m, (size_t)st.st_size, MADV_SEQUENTIAL);
            out.map_ = m;
            out.n_ = (size_t)st.st_size;
            close(fd);
            return out;
        }
    }
    char chunk[1 << 16];
    ssize_t r;
    while ((r = ::read(fd, chunk, sizeof chunk)) > 0) out.buf_.insert(out.buf_.end(), chunk, chunk + r);
    close(fd);
    if (r < 0) throw IoError("cannot read " + path + ": " + strerror(errno));
    return out;
}

struct EdgeChunk {
    std::vector<long long> a, b;
    std::vector<double> w;
};

// Lines of byte range [from, to) (from at a line start), the lines getline
// would give, each read as both loaders read a link line: two integers and an
// optional weight (edge list FileIO.cpp:196-222, Pajek arcs :140-160); `buf`
// is the stream state entering the range. Only the edge list skips '#' lines.
void parse_edge_bytes(const FileBytes &d, size_t from, size_t to, Tok buf, bool skip_comments,
                      EdgeChunk &out) {
    const char *base = d.data();
    size_t s = from;
    auto line = [&](size_t b0, size_t e0) {
        const char *b = base + b0, *e = base + e0;
        if (skip_comments && b < e && *b == '#') return;  // FileIO.cpp:198 (line[0] of "" is '\0')
        LineStream ss(b, e);
        ss.read(buf);
        const long long x = c_atol(buf);
        ss.read(buf);
        const long long y = c_atol(buf);
        buf = Tok();
        ss.read(buf);
        const double w = buf.empty() ? 1.0 : c_atof(buf);
        out.a.push_back(x);
        out.b.push_back(y);
        out.w.push_back(w);
    };
    for (const char *p = base + from, *end = base + to; p < end;) {
        const char *nl = static_cast<const char *>(memchr(p, '\n', (size_t)(end - p)));
        if (!nl) break;
        const size_t i = (size_t)(nl - base);
        line(s, i);
        s = i + 1;
        p = nl + 1;
    }
    if (s < to) line(s, to);
}

// State of `buf` entering the line that starts at byte pos (lo <= pos, both
// line starts): the third token (or "") of the last line before it in
// [lo, pos) that was read (with skip_comments, not a '#' line), else `first`,
// the state entering lo.
Tok state_before_pos(const FileBytes &d, size_t lo, size_t pos, bool skip_comments, Tok first) {
    const char *base = d.data();
    size_t e = pos;  // the previous line ends at e - 1 ('\n')
    while (e > lo) {
        const size_t le = e - 1;  // index of the '\n' ending the previous line
        size_t b = le;
        while (b > lo && base[b - 1] != '\n') b--;
        if (!(skip_comments && b < le && base[b] == '#')) {
            LineStream ss(base + b, base + le);
            Tok t;
            ss.read(t);
            ss.read(t);
            Tok third;
            ss.read(third);
            return third;
        }
        e = b;
    }
    return first;
}

// Threads for a byte range: one below 1 MB, else `threads` (at most 64).
int range_threads(size_t bytes, int threads) {
    return bytes < (size_t(1) << 20) ? 1 : std::max(1, std::min(threads, 64));
}

// [lo, hi) split into T byte ranges that start at line starts.
std::vector<size_t> line_cuts(const FileBytes &d, size_t lo, size_t hi, int T) {
    std::vector<size_t> cut(T + 1, hi);
    cut[0] = lo;
    for (int t = 1; t < T; t++) {
        size_t c = std::max(cut[t - 1], lo + (hi - lo) * t / T);
        while (c < hi && c > lo && d[c - 1] != '\n') c++;
        cut[t] = c;
    }
    return cut;
}

}  // namespace

ParsedGraph parse_edge_list(const std::string &path, int threads) {
    FileBytes d = FileBytes::read(path);
    const int T = range_threads(d.size(), threads);
    const std::vector<size_t> cut = line_cuts(d, 0, d.size(), T);
    std::vector<EdgeChunk> chunks(T);
    std::vector<long long> lo(T, LLONG_MAX), hi(T, LLONG_MIN);
    auto parallel = [&](auto &&job) { run_parallel(T, job); };
    parallel([&](int t) {
        const size_t reserve = (cut[t + 1] - cut[t]) / 16 + 16;
        chunks[t].a.reserve(reserve);
        chunks[t].b.reserve(reserve);
        chunks[t].w.reserve(reserve);
        parse_edge_bytes(d, cut[t], cut[t + 1], state_before_pos(d, 0, cut[t], true, Tok()), true, chunks[t]);
        for (size_t i = 0; i < chunks[t].a.size(); i++) {
            lo[t] = std::min({lo[t], chunks[t].a[i], chunks[t].b[i]});
            hi[t] = std::max({hi[t], chunks[t].a[i], chunks[t].b[i]});
        }
    });
    d.release();
    size_t total = 0;
    long long mn = LLONG_MAX, mx = LLONG_MIN;
    for (int t = 0; t < T; t++) {
        total += chunks[t].a.size();
        mn = std::min(mn, lo[t]);
        mx = std::max(mx, hi[t]);
    }
    // every id seen, renumbered in ascending order (FileIO.cpp:242-255): by a
    // presence table when the ids are dense, else by sorting them
    ParsedGraph g;
    std::vector<long long> ids;
    std::vector<int32_t> table;
    // (the span in unsigned arithmetic: ids may cover the whole 64-bit range)
    const unsigned long long span = (unsigned long long)mx - (unsigned long long)mn;
    const bool dense = total > 0 && span < 4ull * (2 * total) + 1024;
    if (dense) {
        const size_t range = (size_t)span + 1, words = (range + 63) / 64;
        // a presence bitmap per thread (no cache line written by two threads),
        // then OR-ed slice by slice
        std::vector<std::vector<uint64_t>> bits(T);
        parallel([&](int t) {
            bits[t].assign(words, 0);
            uint64_t *b = bits[t].data();
            const EdgeChunk &c = chunks[t];
            for (size_t i = 0; i < c.a.size(); i++) {
                const size_t va = (size_t)c.a[i] - (size_t)mn, vb = (size_t)c.b[i] - (size_t)mn;
                b[va >> 6] |= uint64_t(1) << (va & 63);
                b[vb >> 6] |= uint64_t(1) << (vb & 63);
            }
        });
        parallel([&](int t) {
            const size_t w0 = words * t / T, w1 = words * (t + 1) / T;
            for (int u = 1; u < T; u++)
                for (size_t x = w0; x < w1; x++) bits[0][x] |= bits[u][x];
        });
        table.assign(range, -1);
        int64_t k = 0;
        for (size_t x = 0; x < words; x++)
            for (uint64_t m = bits[0][x]; m; m &= m - 1) {
                const size_t v = x * 64 + (size_t)__builtin_ctzll(m);
                table[v] = (int32_t)k++;
                ids.push_back((long long)((unsigned long long)mn + v));
            }
        if (k >= (int64_t)INT32_MAX) throw FormatError("more than 2^31-1 nodes");
    } else {
        ids.reserve(2 * total);
        for (auto &c : chunks) {
            ids.insert(ids.end(), c.a.begin(), c.a.end());
            ids.insert(ids.end(), c.b.begin(), c.b.end());
        }
        std::sort(ids.begin(), ids.end());
        ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
        if (ids.size() >= (size_t)INT32_MAX) throw FormatError("more than 2^31-1 nodes");
    }
    g.n = (int32_t)ids.size();
    g.n_lines = (int64_t)total;
    g.names.resize(ids.size());
    parallel([&](int t) {
        for (size_t i = ids.size() * t / T; i < ids.size() * (t + 1) / T; i++) g.names[i] = std::to_string(ids[i]);
    });
    auto ren = [&](long long x) -> int32_t {
        if (dense) return table[(size_t)x - (size_t)mn];
        return (int32_t)(std::lower_bound(ids.begin(), ids.end(), x) - ids.begin());
    };
    // non-self links per chunk, then every chunk renumbered into its slice in order
    std::vector<size_t> keep(T + 1, 0);
    parallel([&](int t) {
        size_t k = 0;
        for (size_t i = 0; i < chunks[t].a.size(); i++) k += chunks[t].a[i] != chunks[t].b[i];
        keep[t + 1] = k;
    });
    for (int t = 0; t < T; t++) keep[t + 1] += keep[t];
    g.src.resize(keep[T]);
    g.dst.resize(keep[T]);
    g.w.resize(keep[T]);
    std::vector<std::vector<std::pair<int32_t, double>>> selfs(T);
    parallel([&](int t) {
        size_t o = keep[t];
        const EdgeChunk &c = chunks[t];
        for (size_t i = 0; i < c.a.size(); i++) {
            const int32_t x = ren(c.a[i]);
            if (c.a[i] == c.b[i]) {
                selfs[t].push_back({x, c.w[i]});
                continue;
            }
            g.src[o] = x;
            g.dst[o] = ren(c.b[i]);
            g.w[o] = c.w[i];
            o++;
        }
    });
    std::map<int32_t, double> self;  // summed in input order, as the edge map does
    for (auto &v : selfs)
        for (auto &kv : v) self[kv.first] += kv.second;
    for (auto &kv : self)
        if (kv.second > 0.0) g.n_self++;
    return g;
}

ParsedGraph parse_pajek(const std::string &path, int threads) {
    FileBytes d;
    try {
        d = FileBytes::read(path);
    } catch (const IoError &) {
        // the reference reads from a failed stream: "not in Pajek format"
        throw FormatError("the network file is not in Pajek format...exiting");
    }
    const char *base = d.data();
    size_t pos = 0;  // start of the next getline line; d.size() when there is none
    // the next line, or an empty one past the end (a failed getline reads nothing)
    auto next_line = [&](const char *&b, const char *&e) {
        if (pos >= d.size()) {
            b = e = base;
            return;
        }
        const char *nl = static_cast<const char *>(memchr(base + pos, '\n', d.size() - pos));
        const size_t end = nl ? (size_t)(nl - base) : d.size();
        b = base + pos;
        e = base + end;
        pos = nl ? end + 1 : d.size();
    };
    Tok buf;
    long long n = 0;
    while (n == 0) {  // FileIO.cpp:59-77
        if (pos >= d.size()) throw FormatError("the network file is not in Pajek format...exiting");
        const char *b, *e;
        next_line(b, e);
        LineStream ss(b, e);
        ss.read(buf);
        const std::string t = buf.str();
        if (t == "*Vertices" || t == "*vertices" || t == "*VERTICES") {
            ss.read(buf);
            n = c_atol(buf);
        } else {
            throw FormatError("the network file is not in Pajek format...exiting");
        }
    }
    if (n < 0 || n >= INT32_MAX) throw FormatError("invalid vertex count");
    ParsedGraph g;
    g.n = (int32_t)n;
    g.names.resize((size_t)n);
    g.node_w.assign((size_t)n, 1.0);
    for (long long i = 0; i < n; i++) {  // FileIO.cpp:86-121
        if (pos >= d.size()) throw FormatError("Number of nodes not matching, exiting");
        const char *b, *e;
        next_line(b, e);
        LineStream ss(b, e);
        ss.read(buf);
        const char *q0 = nullptr, *q1 = nullptr;
        for (const char *c = b; c < e; c++)
            if (*c == '"') {
                if (!q0) q0 = c;
                q1 = c;
            }
        LineStream rest(b, e);
        if (q0 && q0 < q1) {
            g.names[i].assign(q0 + 1, q1);
            rest = LineStream(q1 + 1, e);
        } else {
            rest.read(buf);
            rest.read(buf);
            g.names[i] = buf.str();
        }
        static const char one[] = "1";
        buf.b = one;
        buf.e = one + 1;
        rest.read(buf);
        double x = c_atof(buf);
        if (x <= 0.0) x = 1.0;
        g.node_w[i] = x;
    }
    {  // FileIO.cpp:126-134
        const char *b, *e;
        next_line(b, e);
        LineStream ss(b, e);
        ss.read(buf);
        const std::string t = buf.str();
        if (t != "*Edges" && t != "*edges" && t != "*Arcs" && t != "*arcs")
            throw FormatError("Number of nodes not matching, exiting");
    }
    // the link lines (FileIO.cpp:140-160) in byte ranges on all threads: the
    // state entering the first is the header token still in buf
    const size_t lo = pos, hi = d.size();
    const int T = range_threads(hi - lo, threads);
    const std::vector<size_t> cut = line_cuts(d, lo, hi, T);
    std::vector<EdgeChunk> chunks(T);
    const Tok header = buf;
    run_parallel(T, [&](int t) {
        parse_edge_bytes(d, cut[t], cut[t + 1], state_before_pos(d, lo, cut[t], false, header), false, chunks[t]);
    });
    // ids are 1-based; self-links are counted and dropped before the range
    // check (OmpRelaxmap.cpp:123-128); the first link outside 1..n in file
    // order is the error
    auto id0 = [](long long v) { return (long long)((unsigned long long)v - 1ull); };
    std::vector<size_t> keep(T + 1, 0);
    std::vector<int64_t> bad(T, -1);
    run_parallel(T, [&](int t) {
        const EdgeChunk &c = chunks[t];
        size_t k = 0;
        for (size_t i = 0; i < c.a.size(); i++) {
            const long long x = id0(c.a[i]), y = id0(c.b[i]);
            if (x == y) continue;
            if (x < 0 || y < 0 || x >= n || y >= n) {
                bad[t] = (int64_t)i;
                break;
            }
            k++;
        }
        keep[t + 1] = k;
    });
    for (int t = 0; t < T; t++) {
        if (bad[t] >= 0) {
            const size_t i = (size_t)bad[t];
            throw FormatError("link " + std::to_string(chunks[t].a[i]) + " " + std::to_string(chunks[t].b[i]) +
                              " outside 1.." + std::to_string(n));
        }
        keep[t + 1] += keep[t];
        g.n_lines += (int64_t)chunks[t].a.size();
    }
    g.src.resize(keep[T]);
    g.dst.resize(keep[T]);
    g.w.resize(keep[T]);
    std::vector<std::vector<std::pair<long long, double>>> selfs(T);
    run_parallel(T, [&](int t) {
        const EdgeChunk &c = chunks[t];
        size_t o = keep[t];
        for (size_t i = 0; i < c.a.size(); i++) {
            const long long x = id0(c.a[i]), y = id0(c.b[i]);
            if (x == y) {
                selfs[t].push_back({x, c.w[i]});
                continue;
            }
            g.src[o] = (int32_t)x;
            g.dst[o] = (int32_t)y;
            g.w[o] = c.w[i];
            o++;
        }
    });
    std::map<long long, double> self;  // summed in file order
    for (auto &v : selfs)
        for (auto &kv : v) self[kv.first] += kv.second;
    for (auto &kv : self)
        if (kv.second > 0.0) g.n_self++;
    return g;
}

ParsedGraph parse_file(const std::string &path, int threads) {
    const size_t dot = path.find_last_of('.');
    const std::string ext = dot == std::string::npos ? std::string() : path.substr(dot);
    if (ext == ".net") return parse_pajek(path, threads);
    return parse_edge_list(path, threads);
}

namespace {

// Threads for formatting n output lines: one below 100K lines.
int writer_threads(size_t n) {
    if (n < 100000) return 1;
    const unsigned hw = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(hw == 0 ? 1u : hw, 16u));
}

void write_all(FILE *f, const std::vector<std::string> &parts, const std::string &file) {
    for (const std::string &s : parts)
        if (!s.empty() && fwrite(s.data(), 1, s.size(), f) != s.size()) {
            fclose(f);
            throw IoError("cannot write " + file);
        }
}

}  // namespace

void write_tree(const std::string &file, double L_bits, int32_t n_modules, const std::vector<int32_t> &part,
                const std::vector<double> &size, const std::vector<std::string> &names) {
    FILE *f = fopen(file.c_str(), "wb");
    if (!f) throw IoError("cannot write " + file);
    fprintf(f, "# Code length %g in %d modules.\n", L_bits, n_modules);
    const size_t n = part.size();
    // members of each module in node order (updateMembersInModule, Module.cpp:2900-2901),
    // modules in index order, renumbered 1.. over the non-empty ones
    std::vector<int64_t> head(n + 1, 0);
    for (size_t v = 0; v < n; v++) head[(size_t)part[v] + 1]++;
    for (size_t m = 0; m < n; m++) head[m + 1] += head[m];
    std::vector<int32_t> mem(n);
    std::vector<int64_t> fill(head.begin(), head.end() - 1);
    for (size_t v = 0; v < n; v++) mem[fill[(size_t)part[v]]++] = (int32_t)v;
    std::vector<int32_t> modnum(n, 0);
    int32_t mod = 0;
    for (size_t m = 0; m < n; m++)
        if (head[m + 1] > head[m]) modnum[m] = ++mod;
    // the lines of member positions [j0, j1) formatted by each thread, written in order
    const int T = writer_threads(n);
    std::vector<std::string> out(T);
    run_parallel(T, [&](int t) {
        const int64_t j0 = (int64_t)(n * t / T), j1 = (int64_t)(n * (t + 1) / T);
        if (j0 >= j1) return;
        std::string &s = out[t];
        s.reserve((size_t)(j1 - j0) * 40);
        size_t m = (size_t)(std::upper_bound(head.begin(), head.end(), j0) - head.begin()) - 1;
        char line[96];
        for (int64_t j = j0; j < j1; j++) {
            while (head[m + 1] <= j) m++;
            const int32_t v = mem[(size_t)j];
            const int k = snprintf(line, sizeof line, "%d:%lld %g \"", modnum[m], (long long)(j - head[m] + 1),
                                   size[(size_t)v]);
            s.append(line, (size_t)k);
            if (v < (int32_t)names.size()) s.append(names[(size_t)v]);
            s.append("\"\n");
        }
    });
    write_all(f, out, file);
    fclose(f);
}

void write_clu(const std::string &file, const std::vector<int32_t> &part) {
    FILE *f = fopen(file.c_str(), "wb");
    if (!f) throw IoError("cannot write " + file);
    fprintf(f, "*Vertices %zu\r\n", part.size());
    const size_t n = part.size();
    const int T = writer_threads(n);
    std::vector<std::string> out(T);
    run_parallel(T, [&](int t) {
        std::string &s = out[t];
        s.reserve((n / T + 1) * 8);
        char line[24];
        for (size_t i = n * t / T; i < n * (t + 1) / T; i++) {
            const int k = snprintf(line, sizeof line, "%d\r\n", part[i] + 1);
            s.append(line, (size_t)k);
        }
    });
    write_all(f, out, file);
    fclose(f);
}

std::vector<int32_t> read_clu(const std::string &file, int32_t n) {
    FileBytes d = FileBytes::read(file);
    const char *p = d.data(), *end = d.data() + d.size();
    // the next token on the current line, or an empty one at its end
    auto token = [&](const char *&b, const char *&e) {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) p++;
        b = p;
        while (p < end && !is_ws(*p)) p++;
        e = p;
    };
    auto next_line = [&] {
        while (p < end && *p != '\n') p++;
        if (p < end) p++;
    };
    auto integer = [&](const char *b, const char *e, long long &v) {
        if (b == e) return false;
        v = 0;
        for (const char *c = b; c < e; c++) {
            if (*c < '0' || *c > '9' || v > INT32_MAX) return false;
            v = v * 10 + (*c - '0');
        }
        return true;
    };
    const char *b, *e;
    token(b, e);
    const std::string head(b, e);
    if (head != "*Vertices" && head != "*vertices" && head != "*VERTICES")
        throw FormatError(file + ": no *Vertices line");
    token(b, e);
    long long count = 0;
    if (!integer(b, e, count) || count != n)
        throw FormatError(file + ": " + std::string(b, e) + " vertices, the graph has " + std::to_string(n));
    next_line();
    std::vector<int32_t> part((size_t)n);
    for (int32_t i = 0; i < n; i++) {
        token(b, e);
        long long label = 0;
        if (!integer(b, e, label) || label < 1 || label > n)
            throw FormatError(file + ": label of node " + std::to_string(i + 1) + " is not an integer in 1.." +
                              std::to_string(n));
        part[(size_t)i] = (int32_t)(label - 1);
        next_line();
    }
    return part;
}

}  // namespace rmx
