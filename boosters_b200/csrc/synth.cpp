// synth.cpp — the seeded synthetic workloads of synth_gen.h on the C ABI.
#include "synth_gen.h"

#include "../../include/boosters_c.h"

extern "C" {

bst_status bst_synth_regression(uint64_t n, uint64_t F, uint64_t n_inf, uint64_t seed, uint64_t stream,
                                float* x, float* y) {
    return synthgen::regression(n, F, n_inf, seed, stream, x, y) ? BST_ERR_INVALID_ARGUMENT : BST_OK;
}

bst_status bst_synth_binary(uint64_t n, uint64_t F, uint64_t n_nan_cols, uint64_t seed, uint64_t stream,
                            float* x, float* y) {
    return synthgen::binary(n, F, n_nan_cols, seed, stream, x, y) ? BST_ERR_INVALID_ARGUMENT : BST_OK;
}

bst_status bst_synth_multiclass(uint64_t n, uint64_t n_num, uint64_t n_cat, uint64_t C, uint64_t seed,
                                uint64_t stream, float* x, float* y) {
    return synthgen::multiclass(n, n_num, n_cat, C, seed, stream, x, y) ? BST_ERR_INVALID_ARGUMENT : BST_OK;
}

}  // extern "C"
