// specseq_b200.hpp - header-only C++ mirror of the reference's host class over
// the C ABI of sspp.h.
//
// The reference drives its reduction through class SpecSeqPlusPlus
// (include/specseq.h:63-1194): the constructor takes the matrix as the
// vectors processFiles builds (src/main.cu:90-167: a dummy empty column 0,
// face indices shifted by +1), then GPU_Init(), GPU_Compute() and
// GetPersistencePairs() (include/specseq.h:486-512, 513, 592, 1182).  This class
// keeps those names, argument meanings and return values, so swapping
// `#include "specseq.h"` for `#include "specseq_b200.hpp"` in src/main.cu and
// linking libsspp.so replaces the reduction.  Like the reference, a failure
// prints a message and exits with EXIT_FAILURE (include/kernel.h:26-32).
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <utility>
#include <vector>

#include "sspp.h"

class SpecSeqPlusPlus {
public:
    SpecSeqPlusPlus() = default;

    // hv_csc / hv_dim as built by the reference's reader: column 0 is an empty
    // dummy, face indices are shifted by +1.  hv_neighbor is accepted for
    // signature compatibility (the engine builds its own adjacency).
    SpecSeqPlusPlus(std::vector<std::vector<int32_t>>& hv_csc, std::vector<int32_t>& hv_dim,
                    std::vector<std::vector<int32_t>>& hv_neighbor, int32_t* level_capacity, int32_t dualize,
                    int32_t model, int32_t highclear_maxneighbors, int32_t ssBlockSize, float blockSizeGrowthRate,
                    int32_t queuSize) {
        (void)hv_neighbor;
        sspp_default_params(&params_);
        params_.dualize = dualize;
        params_.model = model;
        params_.max_iteration = highclear_maxneighbors;
        params_.ss_block_size = ssBlockSize;
        params_.growth = blockSizeGrowthRate;
        params_.queue_size = queuSize;
        params_.level1_capacity = level_capacity[1];
        params_.level2_capacity = level_capacity[2];
        sspp_config cfg{};
        ctx_ = sspp_create(&cfg);
        if (!ctx_) die("no usable CUDA device");
        // drop the dummy column and undo the +1 shift
        const size_t n = hv_csc.empty() ? 0 : hv_csc.size() - 1;
        std::vector<int32_t> dims(n);
        std::vector<int64_t> col_ptr(n + 1, 0);
        std::vector<int32_t> rows;
        for (size_t j = 0; j < n; j++) {
            dims[j] = hv_dim[j + 1];
            for (int32_t r : hv_csc[j + 1]) rows.push_back(r - 1);
            col_ptr[j + 1] = int64_t(rows.size());
        }
        check(sspp_load_csc(ctx_, int64_t(n), dims.data(), col_ptr.data(), rows.data()));
    }

    SpecSeqPlusPlus(const SpecSeqPlusPlus&) = delete;
    SpecSeqPlusPlus& operator=(const SpecSeqPlusPlus&) = delete;
    ~SpecSeqPlusPlus() {
        if (ctx_) sspp_destroy(ctx_);
    }

    // seconds, as the reference returns them
    float GPU_Init() {
        check(sspp_init(ctx_, &params_, nullptr));
        sspp_stats st;
        sspp_get_stats(ctx_, &st);
        return float(st.init_ms / 1000.0);
    }

    float GPU_Compute() {
        check(sspp_compute(ctx_, nullptr));
        sspp_stats st;
        sspp_get_stats(ctx_, &st);
        return float(st.compute_ms / 1000.0);
    }

    // (birth, death) in the input's 0-based indices, sorted
    std::vector<std::pair<int64_t, int64_t>>& GetPersistencePairs() {
        pairs_.clear();
        const int64_t k = sspp_num_pairs(ctx_);
        if (k < 0) die(sspp_last_error(ctx_));
        std::vector<int64_t> bd(size_t(2 * k));
        if (sspp_pairs(ctx_, bd.data(), k) != k) die(sspp_last_error(ctx_));
        pairs_.reserve(size_t(k));
        for (int64_t i = 0; i < k; i++) pairs_.emplace_back(bd[2 * i], bd[2 * i + 1]);
        return pairs_;
    }

    void setDataFileName(const std::string& name) { name_ = name; }

private:
    [[noreturn]] static void die(const char* msg) {
        std::fprintf(stderr, "CUDA Error: %s\n", msg);
        std::exit(EXIT_FAILURE);
    }
    void check(int32_t rc) {
        if (rc != SSPP_OK) die(sspp_last_error(ctx_));
    }

    sspp_ctx* ctx_ = nullptr;
    sspp_params params_{};
    std::vector<std::pair<int64_t, int64_t>> pairs_;
    std::string name_;
};
