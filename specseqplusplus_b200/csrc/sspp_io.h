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

}  // namespace sspp
