// specseq++ : drop-in command line for the reference's binary (src/main.cu:169-352).
//
//   specseq++ <input_file> <output_file> <ascii|binary> <ascii|binary> <dualize>
//             <model> <max_iteration> <ss_block_size> <block_size_growth_rate>
//             <queue_size> <level1_capacity> <level2_capacity> [--auto] [--device N]
//             [--export-preprocessed]
//
// Same 12 positional arguments, same pair file bytes (count line, then
// "birth death" lines, or int64 count + int64 pairs), same exit codes (0, or 1
// with the help text on bad arguments).  `--auto` lets the engine pick the
// block sizes, queue size and capacities for the input's size class.
// `--export-preprocessed` does what the reference's HIGHOUT build does
// (include/specseq.h:545-549, 1108-1129): it writes the input with the guided
// clearing / edge collapse of <model> applied to <output_file> (in the output
// format) instead of the pairs, and stops.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "sspp.h"

static void print_help() {
    std::printf(
        "Usage: specseq++ <input_file> <output_file> <input_format> <output_format> <dualize> <model> "
        "<max_iteration> <ss_block_size> <block_size_growth_rate> <queue_size> <level1_capacity> "
        "<level2_capacity> [--auto] [--device N] [--export-preprocessed]\n"
        "input_format: ascii or binary\n"
        "output_format: ascii or binary\n"
        "dualize: \n"
        "  0 - No dualize\n"
        "  1 - Enable dualize\n"
        "model: \n"
        "  0 - No optimizations\n"
        "  1 - Enable high-dimensional clearing theorem\n"
        "  2 - Enable edge collapsing\n"
        "  3 - Enable both high-dimension guided clearing theorem and edge collapsing\n"
        "max_iteration[Only effective when model equals 1 or 3.]: candidates examined per top-dimension simplex "
        "by the high-dimension guided clearing\n"
        "ss_block_size: Block size for ss (default 102400)\n"
        "block_size_growth_rate: Block size growth rate (default 1.05)\n"
        "queue_size: maximum number of concurrent column workers (default 65536)\n"
        "level1_capacity: on-chip capacity (ints) of a column worker\n"
        "level2_capacity: on-chip capacity (ints) of a block worker\n"
        "--auto: choose ss_block_size, growth, queue_size and capacities automatically\n"
        "--export-preprocessed: write the input with the model's clearing / collapse applied (cleared columns "
        "as dimension-only lines) to output_file instead of the pairs\n"
        "Example: ./specseq++ input.txt output.txt ascii ascii 0 1 10 1024000 1.05 65536 1000 2000\n");
}

static bool parse_int(const char* s, int32_t& v) {
    char* end = nullptr;
    long x = std::strtol(s, &end, 10);
    if (end == s || x < INT32_MIN || x > INT32_MAX) return false;
    v = int32_t(x);
    return true;
}

static bool parse_float(const char* s, float& v) {
    char* end = nullptr;
    v = std::strtof(s, &end);
    return end != s;
}

int main(int argc, char** argv) {
    if (argc == 2 && (std::strcmp(argv[1], "-help") == 0 || std::strcmp(argv[1], "-h") == 0)) {
        print_help();
        return 0;
    }
    if (argc < 13) {
        std::fprintf(stderr, "Invalid number of arguments.\n");
        print_help();
        return 1;
    }
    const char* in = argv[1];
    const char* out = argv[2];
    int in_fmt, out_fmt;
    if (!std::strcmp(argv[3], "ascii")) in_fmt = SSPP_ASCII;
    else if (!std::strcmp(argv[3], "binary")) in_fmt = SSPP_BINARY;
    else {
        std::fprintf(stderr, "Invalid input format. Format should be 'ascii' or 'binary'.\n");
        print_help();
        return 1;
    }
    if (!std::strcmp(argv[4], "ascii")) out_fmt = SSPP_ASCII;
    else if (!std::strcmp(argv[4], "binary")) out_fmt = SSPP_BINARY;
    else {
        std::fprintf(stderr, "Invalid output format. Format should be 'ascii' or 'binary'.\n");
        print_help();
        return 1;
    }
    sspp_params p;
    sspp_default_params(&p);
    if (!parse_int(argv[5], p.dualize) || !parse_int(argv[6], p.model) || !parse_int(argv[7], p.max_iteration) ||
        !parse_int(argv[8], p.ss_block_size) || !parse_float(argv[9], p.growth) || !parse_int(argv[10], p.queue_size) ||
        !parse_int(argv[11], p.level1_capacity) || !parse_int(argv[12], p.level2_capacity)) {
        std::fprintf(stderr, "Invalid numeric argument.\n");
        print_help();
        return 1;
    }
    sspp_config cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    bool export_only = false;
    for (int i = 13; i < argc; i++) {
        if (!std::strcmp(argv[i], "--auto")) p.autotune = 1;
        else if (!std::strcmp(argv[i], "--export-preprocessed")) export_only = true;
        else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) cfg.device = std::atoi(argv[++i]);
    }
    sspp_ctx* ctx = sspp_create(&cfg);
    if (!ctx) {
        std::fprintf(stderr, "Error: no usable CUDA device.\n");
        return 1;
    }
    int rc = sspp_load_phat(ctx, in, in_fmt);
    if (rc == SSPP_OK) std::printf("-----------------------------------------------Reading  completed-----------------------------------------------\n");
    if (rc == SSPP_OK && export_only) {
        rc = sspp_export_preprocessed(ctx, &p, out, out_fmt);
        if (rc != SSPP_OK) std::fprintf(stderr, "Error: %s\n", sspp_last_error(ctx));
        sspp_destroy(ctx);
        return rc == SSPP_OK ? 0 : 1;
    }
    if (rc == SSPP_OK) rc = sspp_init(ctx, &p, nullptr);
    if (rc == SSPP_OK) rc = sspp_compute(ctx, nullptr);
    if (rc != SSPP_OK) {
        std::fprintf(stderr, "Error: %s\n", sspp_last_error(ctx));
        sspp_destroy(ctx);
        return 1;
    }
    sspp_stats st;
    sspp_get_stats(ctx, &st);
    std::printf("Initialization Time: %10.6f seconds\n", st.init_ms / 1000.0);
    std::printf("Computation    Time: %10.6f seconds\n", st.compute_ms / 1000.0);
    std::printf("Total          Time: %10.6f seconds\n", (st.init_ms + st.compute_ms) / 1000.0);
    rc = sspp_write_pairs(ctx, out, out_fmt);
    if (rc != SSPP_OK) {
        std::fprintf(stderr, "Error: %s\n", sspp_last_error(ctx));
        sspp_destroy(ctx);
        return 1;
    }
    std::printf("-----------------------------------------------Writing  completed-----------------------------------------------\n");
    sspp_destroy(ctx);
    return 0;
}
