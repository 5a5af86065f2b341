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
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sspp_io.h"

namespace sspp {

static bool read_all(const char* path, std::string& buf) {
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

bool read_phat(const char* path, int fmt, PhatMatrix& m, std::string& err) {
    m.dims.clear();
    m.col_ptr.assign(1, 0);
    m.rows.clear();
    std::string buf;
    if (!read_all(path, buf)) {
        err = std::string("cannot read ") + path;
        return false;
    }
    std::vector<int32_t> col;
    if (fmt == 0) {
        const char* p = buf.data();
        const char* end = p + buf.size();
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
                std::sort(col.begin(), col.end());
                col.erase(std::unique(col.begin(), col.end()), col.end());
                m.dims.push_back(int32_t(d));
                m.rows.insert(m.rows.end(), col.begin(), col.end());
                m.col_ptr.push_back(int64_t(m.rows.size()));
            }
            p = eol ? eol + 1 : end;
        }
    } else {
        const char* p = buf.data();
        const char* end = p + buf.size();
        auto rd = [&](int64_t& v) -> bool {
            if (end - p < 8) return false;
            std::memcpy(&v, p, 8);
            p += 8;
            return true;
        };
        int64_t nc = 0;
        if (!rd(nc) || nc < 0) { err = "truncated binary header"; return false; }
        m.dims.reserve(size_t(nc));
        m.col_ptr.reserve(size_t(nc) + 1);
        for (int64_t j = 0; j < nc; j++) {
            int64_t d = 0, k = 0;
            if (!rd(d) || !rd(k) || k < 0 || k > (end - p) / 8) { err = "truncated binary column"; return false; }
            col.resize(size_t(k));
            for (int64_t t = 0; t < k; t++) {
                int64_t x;
                rd(x);
                if (x < INT32_MIN || x > INT32_MAX) { err = "index out of int32 range"; return false; }
                col[size_t(t)] = int32_t(x);
            }
            std::sort(col.begin(), col.end());
            col.erase(std::unique(col.begin(), col.end()), col.end());
            m.dims.push_back(int32_t(d));
            m.rows.insert(m.rows.end(), col.begin(), col.end());
            m.col_ptr.push_back(int64_t(m.rows.size()));
        }
    }
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
        std::string out;
        out.reserve(size_t(npairs) * 16 + 32);
        char tmp[64];
        int k = std::snprintf(tmp, sizeof(tmp), "%lld\n", (long long)npairs);
        out.append(tmp, size_t(k));
        for (int64_t i = 0; i < npairs; i++) {
            k = std::snprintf(tmp, sizeof(tmp), "%lld %lld\n", (long long)bd[2 * i], (long long)bd[2 * i + 1]);
            out.append(tmp, size_t(k));
        }
        ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    } else {
        int64_t n = npairs;
        ok = std::fwrite(&n, 8, 1, f) == 1;
        if (ok && npairs) ok = std::fwrite(bd, 16, size_t(npairs), f) == size_t(npairs);
    }
    if (std::fclose(f) != 0) ok = false;
    if (!ok) err = std::string("write failed: ") + path;
    return ok;
}

}  // namespace sspp
