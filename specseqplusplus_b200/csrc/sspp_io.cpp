// PHAT boundary-matrix reader and persistence-pair writer.
//
// Reader semantics follow processFiles (src/main.cu:90-167): ascii lines are
// right-trimmed; blank lines and lines whose first character is '#' are
// skipped; otherwise the first integer is the column's dimension and the
// following integers are its face indices; parsing of a line stops at the
// first token that is not an integer (a line without a leading integer is an
// empty dimension-0 column, as a failed stream extraction leaves 0 there).
// Binary files hold int64 ncols, then per column int64 dim, int64 count and
// count int64 indices.  Every column is sorted and de-duplicated.  Indices stay
// 0-based (the reference shifts ascii indices by +1 and removes the shift when
// it reports pairs, include/specseq.h:1187; it forgets the shift for binary
// files, src/main.cu:146-155, which this reader does not reproduce).
//
// Writer semantics follow writeVectorToFile (src/main.cu:191-229).
//
// Both run on several host threads for large files: ascii input is cut into
// chunks at line ends and parsed in parallel, binary input is parsed after one
// pass over its column headers, and ascii pair lines are formatted in
// parallel; the results are exactly those of a sequential pass.
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "sspp_io.h"

namespace sspp {

// Read-only view of a whole file: mapped where possible (no copy, pages
// faulted in by the parsing threads), else read into a buffer.
class FileView {
public:
    bool open(const char* path) {
        const int fd = ::open(path, O_RDONLY);
        if (fd < 0) return false;
        struct stat st;
        if (::fstat(fd, &st) != 0) {
            ::close(fd);
            return false;
        }
        size_ = size_t(st.st_size);
        if (size_ > 0) {
            void* m = ::mmap(nullptr, size_, PROT_READ, MAP_PRIVATE, fd, 0);
            if (m != MAP_FAILED) map_ = static_cast<const char*>(m);
        }
        ::close(fd);
        if (size_ > 0 && !map_) return read_all(path, buf_) && (size_ = buf_.size(), true);
        return true;
    }
    ~FileView() {
        if (map_) ::munmap(const_cast<char*>(map_), size_);
    }
    const char* data() const { return map_ ? map_ : buf_.data(); }
    size_t size() const { return size_; }

private:
    static bool read_all(const char* path, std::string& buf);
    const char* map_ = nullptr;
    size_t size_ = 0;
    std::string buf_;
};

bool FileView::read_all(const char* path, std::string& buf) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    if (std::fseek(f, 0, SEEK_END) != 0) { std::fclose(f); return false; }
    long sz = std::ftell(f);
    if (sz < 0) { std::fclose(f); return false; }
    std::fseek(f, 0, SEEK_SET);
    buf.resize(size_t(sz));
    size_t got = sz ? std::fread(&buf[0], 1, size_t(sz), f) : 0;
    std::fclose(f);
    return got == size_t(sz);
}

static inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\f' || c == '\v'; }

// parses one integer token starting at p (leading spaces skipped); false if
// the next token is not an integer that fits int32
static inline bool next_int(const char*& p, const char* end, int64_t& v) {
    while (p < end && is_space(*p)) p++;
    if (p >= end) return false;
    const char* q = p;
    bool neg = false;
    if (*q == '+' || *q == '-') { neg = (*q == '-'); q++; }
    if (q >= end || *q < '0' || *q > '9') return false;
    int64_t x = 0;
    while (q < end && *q >= '0' && *q <= '9') {
        x = x * 10 + (*q - '0');
        if (x > int64_t(INT32_MAX) + 1) return false;
        q++;
    }
    if (q < end && !is_space(*q)) return false;
    v = neg ? -x : x;
    if (v > INT32_MAX || v < INT32_MIN) return false;
    p = q;
    return true;
}

namespace {

// Columns parsed by one thread: dims, local column ends, rows.
struct Chunk {
    std::vector<int32_t> dims;
    std::vector<int64_t> ends;
    std::vector<int32_t> rows;
    bool ok = true;
    std::string err;
};

int reader_threads(size_t bytes) {
    if (bytes < (size_t(4) << 20)) return 1;
    const unsigned hw = std::max(1u, std::min(std::thread::hardware_concurrency(), 16u));
    return int(std::min<size_t>(hw, bytes / (size_t(1) << 20)));
}

template <class F>
void parallel_for(int n, F f) {
    std::vector<std::thread> th;
    for (int t = 1; t < n; t++) th.emplace_back(f, t);
    f(0);
    for (auto& x : th) x.join();
}

// appends column `col` (sorted, de-duplicated) with dimension d
inline void push_col(Chunk& c, int64_t d, std::vector<int32_t>& col) {
    bool strict = true;  // files usually list faces ascending already
    for (size_t i = 1; i < col.size() && strict; i++) strict = col[i - 1] < col[i];
    if (!strict) {
        std::sort(col.begin(), col.end());
        col.erase(std::unique(col.begin(), col.end()), col.end());
    }
    c.dims.push_back(int32_t(d));
    c.rows.insert(c.rows.end(), col.begin(), col.end());
    c.ends.push_back(int64_t(c.rows.size()));
}

void parse_ascii(const char* p, const char* end, Chunk& c) {
    std::vector<int32_t> col;
    const size_t bytes = size_t(end - p);
    c.dims.reserve(bytes / 16 + 16);
    c.ends.reserve(bytes / 16 + 16);
    c.rows.reserve(bytes / 6 + 16);
    while (p < end) {
        const char* eol = static_cast<const char*>(std::memchr(p, '\n', size_t(end - p)));
        const char* le = eol ? eol : end;
        const char* te = le;
        while (te > p && is_space(te[-1])) te--;
        if (te > p && p[0] != '#') {
            const char* q = p;
            int64_t d = 0;
            col.clear();
            if (next_int(q, te, d)) {
                int64_t x;
                while (next_int(q, te, x)) col.push_back(int32_t(x));
            } else {
                d = 0;
            }
            push_col(c, d, col);
        }
        p = eol ? eol + 1 : end;
    }
}

// binary columns [j0, j1) whose data start at the given byte offsets
void parse_binary(const char* base, const std::vector<int64_t>& at, const std::vector<int64_t>& dim,
                  const std::vector<int64_t>& cnt, int64_t j0, int64_t j1, Chunk& c) {
    std::vector<int32_t> col;
    for (int64_t j = j0; j < j1 && c.ok; j++) {
        col.resize(size_t(cnt[size_t(j)]));
        const char* p = base + at[size_t(j)];
        for (int64_t t = 0; t < cnt[size_t(j)]; t++) {
            int64_t x;
            std::memcpy(&x, p + 8 * t, 8);
            if (x < INT32_MIN || x > INT32_MAX) {
                c.ok = false;
                c.err = "index out of int32 range";
                break;
            }
            col[size_t(t)] = int32_t(x);
        }
        push_col(c, dim[size_t(j)], col);
    }
}

// concatenates the chunks in order
void gather(std::vector<Chunk>& ch, PhatMatrix& m) {
    const size_t T = ch.size();
    std::vector<int64_t> c0(T + 1, 0), r0(T + 1, 0);
    for (size_t t = 0; t < T; t++) {
        c0[t + 1] = c0[t] + int64_t(ch[t].dims.size());
        r0[t + 1] = r0[t] + int64_t(ch[t].rows.size());
    }
    m.dims.resize(size_t(c0[T]));
    m.col_ptr.assign(size_t(c0[T]) + 1, 0);
    m.rows.resize(size_t(r0[T]));
    parallel_for(int(T), [&](int t) {
        const Chunk& c = ch[size_t(t)];
        if (!c.dims.empty()) std::memcpy(&m.dims[size_t(c0[t])], c.dims.data(), 4 * c.dims.size());
        if (!c.rows.empty()) std::memcpy(&m.rows[size_t(r0[t])], c.rows.data(), 4 * c.rows.size());
        for (size_t i = 0; i < c.ends.size(); i++) m.col_ptr[size_t(c0[t]) + i + 1] = r0[t] + c.ends[i];
    });
}

// fast decimal formatting of "a b\n"
inline char* put_int(char* o, long long v) {
    char tmp[24];
    int k = 0;
    const bool neg = v < 0;
    unsigned long long u = neg ? 0ull - (unsigned long long)v : (unsigned long long)v;
    do {
        tmp[k++] = char('0' + u % 10);
        u /= 10;
    } while (u);
    if (neg) *o++ = '-';
    while (k) *o++ = tmp[--k];
    return o;
}

}  // namespace

bool read_phat(const char* path, int fmt, PhatMatrix& m, std::string& err) {
    m.dims.clear();
    m.col_ptr.assign(1, 0);
    m.rows.clear();
    FileView file;
    if (!file.open(path)) {
        err = std::string("cannot read ") + path;
        return false;
    }
    const char* data = file.data();
    const size_t sz = file.size();
    if (fmt == 0) {
        // chunks cut after line ends, parsed in parallel
        const int T = reader_threads(sz);
        std::vector<size_t> cut(static_cast<size_t>(T) + 1, sz);
        cut[0] = 0;
        for (int t = 1; t < T; t++) {
            size_t pos = std::max(cut[size_t(t) - 1], sz * size_t(t) / size_t(T));
            const void* nl = pos < sz ? std::memchr(data + pos, '\n', sz - pos) : nullptr;
            cut[size_t(t)] = nl ? size_t(static_cast<const char*>(nl) - data) + 1 : sz;
        }
        std::vector<Chunk> ch(static_cast<size_t>(T));
        parallel_for(T, [&](int t) { parse_ascii(data + cut[size_t(t)], data + cut[size_t(t) + 1], ch[size_t(t)]); });
        gather(ch, m);
        return true;
    }
    // binary: one pass over the column headers, then the columns in parallel
    const char* p = data;
    const char* end = data + sz;
    auto rd = [&](int64_t& v) -> bool {
        if (end - p < 8) return false;
        std::memcpy(&v, p, 8);
        p += 8;
        return true;
    };
    int64_t nc = 0;
    if (!rd(nc) || nc < 0 || nc > int64_t(sz / 16)) {
        err = "truncated binary header";
        return false;
    }
    std::vector<int64_t> at(static_cast<size_t>(nc)), dim(static_cast<size_t>(nc)), cnt(static_cast<size_t>(nc));
    for (int64_t j = 0; j < nc; j++) {
        int64_t d = 0, k = 0;
        if (!rd(d) || !rd(k) || k < 0 || k > (end - p) / 8) {
            err = "truncated binary column";
            return false;
        }
        dim[size_t(j)] = d;
        cnt[size_t(j)] = k;
        at[size_t(j)] = int64_t(p - data);
        p += 8 * k;
    }
    const int T = reader_threads(sz);
    std::vector<Chunk> ch(static_cast<size_t>(T));
    parallel_for(T, [&](int t) {
        parse_binary(data, at, dim, cnt, nc * t / T, nc * (t + 1) / T, ch[size_t(t)]);
    });
    for (auto& c : ch)
        if (!c.ok) {
            err = c.err;
            return false;
        }
    gather(ch, m);
    return true;
}

bool write_pairs(const char* path, int fmt, const int64_t* bd, int64_t npairs, std::string& err) {
    FILE* f = std::fopen(path, fmt == 0 ? "w" : "wb");
    if (!f) {
        err = std::string("could not open file ") + path;
        return false;
    }
    bool ok = true;
    if (fmt == 0) {
        // the pair lines formatted in parallel, written in order
        const int T = reader_threads(size_t(npairs) * 16);
        std::vector<std::string> part(static_cast<size_t>(T));
        parallel_for(T, [&](int t) {
            const int64_t a = npairs * t / T, b = npairs * (t + 1) / T;
            std::string& o = part[size_t(t)];
            o.resize(size_t(b - a) * 42 + 1);
            char* q = &o[0];
            for (int64_t i = a; i < b; i++) {
                q = put_int(q, (long long)bd[2 * i]);
                *q++ = ' ';
                q = put_int(q, (long long)bd[2 * i + 1]);
                *q++ = '\n';
            }
            o.resize(size_t(q - &o[0]));
        });
        char head[32];
        char* q = put_int(head, (long long)npairs);
        *q++ = '\n';
        ok = std::fwrite(head, 1, size_t(q - head), f) == size_t(q - head);
        for (auto& o : part)
            if (ok && !o.empty()) ok = std::fwrite(o.data(), 1, o.size(), f) == o.size();
    } else {
        int64_t n = npairs;
        ok = std::fwrite(&n, 8, 1, f) == 1;
        if (ok && npairs) ok = std::fwrite(bd, 16, size_t(npairs), f) == size_t(npairs);
    }
    if (std::fclose(f) != 0) ok = false;
    if (!ok) err = std::string("write failed: ") + path;
    return ok;
}

bool write_phat(const char* path, int fmt, int64_t ncols, const int32_t* dims, const int64_t* col_ptr,
                const int32_t* rows, std::string& err) {
    FILE* f = std::fopen(path, fmt == 0 ? "w" : "wb");
    if (!f) {
        err = std::string("could not open file ") + path;
        return false;
    }
    bool ok = true;
    const int T = reader_threads(size_t(col_ptr[ncols]) * 8 + size_t(ncols) * 4);
    std::vector<std::string> part(static_cast<size_t>(T));
    parallel_for(T, [&](int t) {
        const int64_t a = ncols * t / T, b = ncols * (t + 1) / T;
        std::string& o = part[size_t(t)];
        if (fmt == 0) {
            o.resize(size_t(col_ptr[b] - col_ptr[a]) * 12 + size_t(b - a) * 13 + 1);
            char* q = &o[0];
            for (int64_t j = a; j < b; j++) {
                q = put_int(q, dims[j]);
                for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; k++) {
                    *q++ = ' ';
                    q = put_int(q, rows[k]);
                }
                *q++ = '\n';
            }
            o.resize(size_t(q - &o[0]));
        } else {
            o.resize(size_t(col_ptr[b] - col_ptr[a] + 2 * (b - a)) * 8);
            char* q = &o[0];
            for (int64_t j = a; j < b; j++) {
                const int64_t h[2] = {dims[j], col_ptr[j + 1] - col_ptr[j]};
                std::memcpy(q, h, 16);
                q += 16;
                for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; k++) {
                    const int64_t x = rows[k];
                    std::memcpy(q, &x, 8);
                    q += 8;
                }
            }
        }
    });
    if (fmt != 0) ok = std::fwrite(&ncols, 8, 1, f) == 1;
    for (auto& o : part)
        if (ok && !o.empty()) ok = std::fwrite(o.data(), 1, o.size(), f) == o.size();
    if (std::fclose(f) != 0) ok = false;
    if (!ok) err = std::string("write failed: ") + path;
    return ok;
}

}  // namespace sspp
