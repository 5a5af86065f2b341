#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace sspp {

struct PhatMatrix {
    std::vector<int32_t> dims;
    std::vector<int64_t> col_ptr;
    std::vector<int32_t> rows;
};

// fmt: 0 ascii, 1 binary
bool read_phat(const char* path, int fmt, PhatMatrix& m, std::string& err);
bool write_pairs(const char* path, int fmt, const int64_t* birth_death, int64_t npairs, std::string& err);
// boundary matrix in PHAT format (ascii: "dim face face ..." lines; binary:
// int64 ncols, then per column int64 dim, int64 count, count int64 faces)
bool write_phat(const char* path, int fmt, int64_t ncols, const int32_t* dims, const int64_t* col_ptr,
                const int32_t* rows, std::string& err);

}  // namespace sspp
