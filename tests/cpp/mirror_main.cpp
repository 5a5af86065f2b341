// Drives the header-only SpecSeqPlusPlus mirror the way the reference's main
// does (src/main.cu:324-349): reader-style vectors with a dummy column 0 and
// +1-shifted indices, GPU_Init, GPU_Compute, GetPersistencePairs.  Reads a PHAT
// ascii file, prints "count" then "birth death" lines.
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "specseq_b200.hpp"

int main(int argc, char** argv) {
    if (argc < 2) return 1;
    std::ifstream in(argv[1]);
    std::vector<std::vector<int32_t>> csc(1);
    std::vector<int32_t> dim(1, 0);
    std::vector<std::vector<int32_t>> nbr;
    std::string line;
    while (std::getline(in, line)) {
        line.erase(line.find_last_not_of(" \t\r\n") + 1);
        if (line.empty() || line[0] == '#') continue;
        std::stringstream ss(line);
        int32_t d, x;
        ss >> d;
        std::vector<int32_t> col;
        while (ss >> x) col.push_back(x + 1);
        csc.push_back(col);
        dim.push_back(d);
    }
    int32_t caps[4] = {0, 1000, 8000, 0};
    SpecSeqPlusPlus alg(csc, dim, nbr, caps, 0, 0, 0, 102400, 1.05f, 65536);
    alg.setDataFileName("mirror");
    float ti = alg.GPU_Init();
    float tc = alg.GPU_Compute();
    auto& pairs = alg.GetPersistencePairs();
    std::printf("%zu\n", pairs.size());
    for (auto& p : pairs) std::printf("%lld %lld\n", (long long)p.first, (long long)p.second);
    std::fprintf(stderr, "init %f compute %f\n", ti, tc);
    return 0;
}
