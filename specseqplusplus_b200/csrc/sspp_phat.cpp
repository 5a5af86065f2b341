// Host-side PHAT file access over the C ABI (include/sspp.h): read a boundary
// matrix into host arrays and write one, without a GPU.  The reader is the
// one sspp_load_phat uses (src/main.cu:90-167 semantics, see sspp_io.cpp).
#include <cstring>
#include <new>
#include <string>

#include "../../include/sspp.h"
#include "sspp_io.h"

struct sspp_phat {
    sspp::PhatMatrix m;
};

namespace {
void put_err(char* err, int32_t cap, const std::string& msg) {
    if (err && cap > 0) {
        std::strncpy(err, msg.c_str(), size_t(cap) - 1);
        err[cap - 1] = 0;
    }
}
}  // namespace

extern "C" {

sspp_phat* sspp_phat_read(const char* path, int32_t fmt, char* err, int32_t err_cap) {
    if (!path || (fmt != SSPP_ASCII && fmt != SSPP_BINARY)) {
        put_err(err, err_cap, "bad path or format");
        return nullptr;
    }
    auto* h = new (std::nothrow) sspp_phat;
    if (!h) return nullptr;
    std::string e;
    if (!sspp::read_phat(path, fmt, h->m, e)) {
        put_err(err, err_cap, e);
        delete h;
        return nullptr;
    }
    return h;
}

int64_t sspp_phat_ncols(const sspp_phat* h) { return h ? int64_t(h->m.dims.size()) : -1; }
int64_t sspp_phat_nnz(const sspp_phat* h) { return h ? int64_t(h->m.rows.size()) : -1; }

int32_t sspp_phat_copy(const sspp_phat* h, int32_t* dims, int64_t* col_ptr, int32_t* rows) {
    if (!h) return SSPP_ERR_BAD_INPUT;
    const auto& m = h->m;
    if (dims && !m.dims.empty()) std::memcpy(dims, m.dims.data(), 4 * m.dims.size());
    if (col_ptr) std::memcpy(col_ptr, m.col_ptr.data(), 8 * m.col_ptr.size());
    if (rows && !m.rows.empty()) std::memcpy(rows, m.rows.data(), 4 * m.rows.size());
    return SSPP_OK;
}

void sspp_phat_free(sspp_phat* h) { delete h; }

int32_t sspp_phat_write(const char* path, int32_t fmt, int64_t ncols, const int32_t* dims, const int64_t* col_ptr,
                        const int32_t* rows, char* err, int32_t err_cap) {
    if (!path || (fmt != SSPP_ASCII && fmt != SSPP_BINARY) || ncols < 0 || !col_ptr || (ncols > 0 && !dims) ||
        (col_ptr[ncols] > 0 && !rows)) {
        put_err(err, err_cap, "bad arguments");
        return SSPP_ERR_BAD_INPUT;
    }
    std::string e;
    if (!sspp::write_phat(path, fmt, ncols, dims, col_ptr, rows, e)) {
        put_err(err, err_cap, e);
        return SSPP_ERR_IO;
    }
    return SSPP_OK;
}

}  // extern "C"
