// binning.h — the plan of feature binning: per-feature analysis, mappers and
// the binned layout (data/binned/feature_analysis.rs:313-569,
// data/binned/dataset.rs:592-750). Numeric bounds and the bins themselves
// are computed on the GPU (kernels.h: launch_numeric_bounds, K1).
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/boosters_c.h"

namespace bst {

enum MissingType : int { MISSING_NONE = 0, MISSING_ZERO = 1, MISSING_NAN = 2 };

// BinMapper (data/binned/bin_mapper.rs:55-271).
struct Mapper {
    bool categorical = false;
    int missing = MISSING_NONE;
    uint32_t n_bins = 0;
    uint32_t default_bin = 0;
    std::vector<double> bounds;  // numeric upper bounds
    std::vector<int32_t> cats;   // categorical: bin -> category (sorted)

    double bin_to_value(uint32_t bin) const {
        return categorical ? (double)cats[bin] : bounds[bin];
    }
    // bins searched by value_to_bin (bin_mapper.rs:237-243)
    uint32_t n_search() const {
        size_t hi = bounds.empty() ? 0 : bounds.size() - 1;
        if (missing == MISSING_NAN) hi = hi == 0 ? 0 : hi - 1;
        return (uint32_t)hi;
    }
};

// Feature layout of a binned dataset: effective columns (non-trivial
// features in original order, data/binned/dataset.rs:460-524) and their
// placement in the u8 / u16 row-major bin matrices.
struct BinPlan {
    uint64_t n = 0;
    uint32_t n_features = 0;
    std::vector<Mapper> mappers;  // per original feature
    std::vector<uint8_t> trivial; // per original feature
    std::vector<uint32_t> col_feature, col_nbins, col_hist_off, col_default, col_matrix, col_pos;
    std::vector<uint8_t> col_cat, col_missing;
    uint32_t f8 = 0, f16 = 0;  // columns per matrix
    // Row record (binning.cpp): rec bytes per row, u8 columns at bytes
    // [0, f8), u16 columns at [u16_off, u16_off + 2 f16). The two matrices
    // are views of it: bins8 = record (stride s8 = rec bytes), bins16 =
    // record + u16_off (stride s16 = rec / 2 elements).
    uint32_t u16_off = 0, rec = 0;
    uint32_t s8 = 0, s16 = 0;
    uint32_t total_bins = 0;
    uint32_t n_cols() const { return (uint32_t)col_feature.size(); }
};

// Bounds of the numeric features, computed off the host (the engine's
// device sort): start() gets the ascending row sample (empty: every row)
// and the features with their NaN flags and may return before the bounds
// are known; finish() stores each feature's mapper into mappers[feature].
struct NumericBounds {
    virtual ~NumericBounds() = default;
    virtual void start(const std::vector<uint32_t>& sample, const std::vector<uint32_t>& features,
                       const std::vector<uint8_t>& has_nan, uint32_t max_bins) = 0;
    virtual void finish(std::vector<Mapper>& mappers) = 0;
};

// The numeric mapper of a feature from its bounds as NumericBounds
// computes them (bin_mapper.rs:55-271: a NaN bin when the feature has NaN
// and two or more distinct finite values).
Mapper numeric_mapper_from_bounds(const double* bounds, uint32_t n_bounds, bool has_nan);

// Analysis + bounds. Returns BST_OK or an error status with `err` set.
// Numeric features' bounds come from `numeric` while the host builds the
// categorical features' mappers.
bst_status plan_binning(const float* x_fm, uint64_t n_features, uint64_t n,
                        const std::vector<uint8_t>& user_categorical, const bst_config& cfg,
                        NumericBounds& numeric, BinPlan& plan, std::string& err);

// Largest f32 <= d (the f32 comparison key equivalent to `v <= d` in f64).
float f32_round_down(double d);

}  // namespace bst
