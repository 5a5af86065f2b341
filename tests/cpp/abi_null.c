/* Compiled as C99 against include/sspp.h and run without a GPU: every entry
 * point given a null context or server returns an error code instead of
 * crashing (the engine checks its handles before any CUDA call). */
#include <stdio.h>

#include "sspp.h"

#define EXPECT(cond)                                           \
    do {                                                       \
        if (!(cond)) {                                         \
            fprintf(stderr, "failed: %s (line %d)\n", #cond, __LINE__); \
            return 1;                                          \
        }                                                      \
    } while (0)

int main(void) {
    float pts[6] = {0, 0, 0, 1, 1, 1};
    float field[8] = {0};
    int64_t out[4];
    int64_t n = 0, nnz = 0;
    sspp_params p;
    sspp_default_params(&p);
    EXPECT(p.representatives == 0 && p.dualize == 0);
    EXPECT(sspp_load_rips(NULL, 2, 3, pts, 0.5f, 3) == SSPP_ERR_BAD_INPUT);
    EXPECT(sspp_load_lowerstar(NULL, 2, 2, 2, field, 3) == SSPP_ERR_BAD_INPUT);
    EXPECT(sspp_input_size(NULL, &n, &nnz) == SSPP_ERR_BAD_INPUT);
    EXPECT(sspp_input_copy(NULL, NULL, NULL, NULL, NULL) == SSPP_ERR_BAD_INPUT);
    EXPECT(sspp_representative(NULL, 0, out, 4) == -1);
    EXPECT(sspp_reduce(NULL, &p, NULL) == SSPP_ERR_BAD_INPUT);
    EXPECT(sspp_server_submit_rips(NULL, 2, 3, pts, 0.5f, 3, 0) == -SSPP_ERR_BAD_INPUT);
    EXPECT(sspp_server_submit_lowerstar(NULL, 2, 2, 2, field, 3, SSPP_SUBMIT_VALUES) == -SSPP_ERR_BAD_INPUT);
    EXPECT(sspp_server_values(NULL, 0, NULL, 0) == -1);
    printf("ok\n");
    return 0;
}
