// oracle.cpp — CPU restatement of egordm/boosters' GBDT hot path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine. The engine
// never links or calls this file. Every block cites the Rust function it
// restates as crates/boosters/src/<file>:<line>.
//
// Build flags matter: -ffp-contract=off (Rust/LLVM never fuses a*b+c) and
// no -ffast-math, so every f32/f64 operation rounds exactly as in Rust.

#include "oracle.h"

// The seeded workload generator, compiled into this library as its own copy
// (a process that runs only the checker never loads the engine).
#include "../boosters_b200/csrc/synth_gen.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;

// ---------------------------------------------------------------------------
// Rust numeric-cast helpers
// ---------------------------------------------------------------------------

// `f64 as f32`: round to nearest even, overflow to +-inf (IEEE conversion).
inline float f64_to_f32(double d) {
    const double lim = 0x1.ffffffp127;  // FLT_MAX + half an ulp: ties round to inf
    const double fmax = (double)std::numeric_limits<float>::max();
    if (d >= lim) return std::numeric_limits<float>::infinity();
    if (d <= -lim) return -std::numeric_limits<float>::infinity();
    if (d > fmax) return std::numeric_limits<float>::max();
    if (d < -fmax) return -std::numeric_limits<float>::max();
    return (float)d;
}

// `f64 as i32` / `f32 as i32`: truncate, saturate, NaN -> 0.
inline int32_t sat_i32(double v) {
    if (std::isnan(v)) return 0;
    if (v >= 2147483647.0) return 2147483647;
    if (v <= -2147483648.0) return (int32_t)-2147483648LL;
    return (int32_t)v;
}

// `f32 as usize`: truncate, negative / NaN -> 0.
inline uint64_t sat_usize(double v) {
    if (std::isnan(v) || v <= 0.0) return 0;
    if (v >= 18446744073709551615.0) return UINT64_MAX;
    return (uint64_t)v;
}

// `f32 as u32` (repr/gbdt/categories.rs:124 float_to_category).
inline uint32_t sat_u32(float v) {
    if (std::isnan(v) || v <= 0.0f) return 0;
    if (v >= 4294967295.0f) return UINT32_MAX;
    return (uint32_t)v;
}

// f32::next_up (training/gbdt/grower.rs:543-556).
inline float next_up_f32(float x) {
    if (std::isnan(x) || x == std::numeric_limits<float>::infinity()) return x;
    if (x == 0.0f) {
        uint32_t one = 1;
        float r;
        std::memcpy(&r, &one, 4);
        return r;
    }
    uint32_t bits;
    std::memcpy(&bits, &x, 4);
    bits = (x > 0.0f) ? bits + 1 : bits - 1;
    float r;
    std::memcpy(&r, &bits, 4);
    return r;
}

// ---------------------------------------------------------------------------
// BinMapper (data/binned/bin_mapper.rs:55-271)
// ---------------------------------------------------------------------------

enum { MISSING_NONE = 0, MISSING_ZERO = 1, MISSING_NAN = 2 };

struct BinMapper {
    std::vector<double> bounds;    // numeric upper bounds
    std::vector<int32_t> cats;     // categorical: bin -> category
    std::unordered_map<int32_t, uint32_t> cat_to_bin;
    uint32_t n_bins = 0;
    int missing = MISSING_NONE;
    uint32_t default_bin = 0;
    bool categorical = false;

    static BinMapper numerical(std::vector<double> b, int missing, uint32_t default_bin) {
        BinMapper m;
        m.bounds = std::move(b);
        m.n_bins = (uint32_t)m.bounds.size();
        m.missing = missing;
        m.default_bin = default_bin;
        return m;
    }
    static BinMapper categorical_from(std::vector<int32_t> c, int missing, uint32_t default_bin) {
        BinMapper m;
        m.categorical = true;
        m.n_bins = (uint32_t)c.size();
        for (size_t i = 0; i < c.size(); ++i) m.cat_to_bin[c[i]] = (uint32_t)i;
        m.cats = std::move(c);
        m.missing = missing;
        m.default_bin = default_bin;
        return m;
    }

    // bin_mapper.rs:210-231
    uint32_t value_to_bin(double value) const {
        if (std::isnan(value)) return missing == MISSING_NAN ? n_bins - 1 : default_bin;
        if (value == 0.0 && missing == MISSING_ZERO) return default_bin;
        if (categorical) {
            auto it = cat_to_bin.find(sat_i32(value));
            return it == cat_to_bin.end() ? 0u : it->second;
        }
        return search_bin(value);
    }
    // bin_mapper.rs:235-258
    uint32_t search_bin(double value) const {
        size_t lo = 0;
        size_t hi = bounds.empty() ? 0 : bounds.size() - 1;
        if (missing == MISSING_NAN) hi = hi == 0 ? 0 : hi - 1;
        while (lo < hi) {
            size_t mid = lo + (hi - lo) / 2;
            if (value <= bounds[mid])
                hi = mid;
            else
                lo = mid + 1;
        }
        return (uint32_t)lo;
    }
    // bin_mapper.rs:261-271
    double bin_to_value(uint32_t bin) const {
        if (categorical) return (double)cats[bin];
        return bounds[bin];
    }
};

// ---------------------------------------------------------------------------
// Feature analysis (data/binned/feature_analysis.rs:313-432, 469-569)
// ---------------------------------------------------------------------------

struct FloatKeyHash {
    size_t operator()(float v) const {
        if (v == 0.0f) v = 0.0f;  // -0.0 == 0.0 under PartialEq
        uint32_t b;
        std::memcpy(&b, &v, 4);
        return std::hash<uint32_t>()(b);
    }
};
struct FloatKeyEq {
    bool operator()(float a, float b) const { return a == b; }
};

struct Analysis {
    bool is_numeric = true, is_sparse = false, needs_u16 = false, is_trivial = true;
    size_t n_unique = 0, n_nonzero = 0, n_valid = 0, n_nan = 0;
    double density = 0.0;
};

Analysis analyze_feature(const float* col, uint64_t n, const bst_config& cfg, bool user_cat) {
    // FeatureStats::new / update (feature_analysis.rs:296-346)
    size_t max_unique = std::max<size_t>(cfg.max_categorical_cardinality, cfg.max_bins) + 10;
    size_t non_zero = 0, valid = 0, nan = 0;
    bool all_int = true, exceeded = false;
    std::unordered_set<float, FloatKeyHash, FloatKeyEq> uniq;
    float first_unique = 0.0f;
    for (uint64_t i = 0; i < n; ++i) {
        float v = col[i];
        if (std::isnan(v)) {
            ++nan;
            continue;
        }
        ++valid;
        if (v != 0.0f) ++non_zero;
        if (all_int) {
            float fr = v - std::trunc(v);  // f32::fract (NaN for +-inf)
            if (!(fr == 0.0f)) all_int = false;
        }
        if (!exceeded && uniq.find(v) == uniq.end()) {
            if (uniq.size() >= max_unique)
                exceeded = true;
            else {
                if (uniq.empty()) first_unique = v;
                uniq.insert(v);
            }
        }
    }
    // FeatureStats::into_analysis (feature_analysis.rs:349-432)
    Analysis a;
    a.n_unique = uniq.size();
    a.n_nonzero = non_zero;
    a.n_valid = valid;
    a.n_nan = nan;
    a.is_trivial = valid == 0 || (a.n_unique == 1 && first_unique == 0.0f) || a.n_unique == 0;
    bool is_binary = a.n_unique == 2;
    bool auto_cat = !user_cat && all_int && a.n_unique <= cfg.max_categorical_cardinality;
    a.is_numeric = user_cat ? false : (is_binary ? true : !auto_cat);
    bool has_nan = nan > 0;
    uint32_t required;
    if (a.is_trivial)
        required = 1;
    else
        required = std::min<uint32_t>((uint32_t)std::min<size_t>(a.n_unique, UINT32_MAX), cfg.max_bins) + (has_nan ? 1 : 0);
    a.needs_u16 = required > 256;
    float density = n == 0 ? 0.0f : (float)non_zero / (float)n;
    a.is_sparse = density <= (1.0f - cfg.sparsity_threshold);
    a.density = n == 0 ? 0.0 : (double)non_zero / (double)n;
    return a;
}

// dataset.rs:598-633 sample_indices_for_binning
std::vector<uint32_t> sample_indices(uint64_t n, uint64_t sample_cnt) {
    std::vector<uint32_t> idx;
    if (n <= sample_cnt) return idx;
    uint64_t k = std::min(sample_cnt, n);
    idx.reserve(k);
    std::unordered_set<uint32_t> seen;
    seen.reserve(k * 2);
    uint64_t state = 0xD1B54A32D192ED03ULL ^ n;
    while (idx.size() < k) {
        state += 0x9E3779B97F4A7C15ULL;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z = z ^ (z >> 31);
        uint32_t i = (uint32_t)(z % n);
        if (seen.insert(i).second) idx.push_back(i);
    }
    std::sort(idx.begin(), idx.end());
    return idx;
}

// dataset.rs:683-750 bin_numeric
BinMapper bin_numeric(const std::vector<float>& data, uint32_t max_bins, bool has_nan) {
    float min_v = std::numeric_limits<float>::max();
    float max_v = -std::numeric_limits<float>::max();
    std::vector<float> values;
    values.reserve(data.size());
    for (float v : data) {
        if (std::isfinite(v)) {
            min_v = std::min(min_v, v);
            max_v = std::max(max_v, v);
            values.push_back(v);
        }
    }
    size_t n_valid = values.size();
    if (n_valid == 0 || min_v >= max_v)
        return BinMapper::numerical({std::numeric_limits<double>::max()}, MISSING_NONE, 0);
    uint32_t n_bins = (uint32_t)std::min<uint64_t>(max_bins, n_valid);
    std::stable_sort(values.begin(), values.end(), [](float a, float b) { return a < b; });
    values.erase(std::unique(values.begin(), values.end(), [](float a, float b) { return a == b; }),
                 values.end());
    size_t n_unique = values.size();
    std::vector<double> bounds;
    if (n_unique <= n_bins) {
        for (size_t i = 0; i + 1 < n_unique; ++i)
            bounds.push_back(((double)values[i] + (double)values[i + 1]) / 2.0);
    } else {
        for (uint32_t i = 1; i < n_bins; ++i) {
            double q = (double)i / (double)n_bins;
            size_t idx = std::min<size_t>((size_t)std::floor(q * (double)(n_unique - 1)), n_unique - 2);
            double bound = ((double)values[idx] + (double)values[idx + 1]) / 2.0;
            if (bounds.empty() || bound > bounds.back()) bounds.push_back(bound);
        }
    }
    bounds.push_back(std::numeric_limits<double>::max());
    if (has_nan) bounds.push_back(std::numeric_limits<double>::max());
    uint32_t nb = (uint32_t)bounds.size();
    return BinMapper::numerical(std::move(bounds), has_nan ? MISSING_NAN : MISSING_NONE,
                                has_nan ? nb - 1 : 0);
}

}  // namespace

// ---------------------------------------------------------------------------
// BinnedDataset (data/binned/dataset.rs:207-309, 460-524)
// ---------------------------------------------------------------------------

struct orc_binned {
    uint64_t n = 0;
    uint32_t n_features = 0;
    std::vector<BinMapper> mappers;
    // effective columns: non-trivial features in original order
    std::vector<uint32_t> col_feature, col_nbins, col_default, col_offset;
    std::vector<uint8_t> col_cat, col_missing;
    std::vector<std::vector<uint16_t>> col_bins;
    uint32_t total_bins = 0;
};

// Per-feature work (analysis, bin mappers, bin assignment) is independent
// across features, so `omp` threads split the features without changing any
// result; the reference runs these loops over rayon the same way.
static int build_binned(const float* x, uint64_t F, uint64_t n, const uint32_t* cat_idx,
                        uint32_t n_cat, const bst_config& cfg, orc_binned& b, int omp = 1) {
    if (omp < 1) omp = 1;
    if (n == 0 || F == 0) {
        g_err = "dataset is empty";
        return BST_ERR_EMPTY_DATASET;
    }
    std::vector<bool> user_cat(F, false);
    for (uint32_t i = 0; i < n_cat; ++i)
        if (cat_idx[i] < F) user_cat[cat_idx[i]] = true;
    b.n = n;
    b.n_features = (uint32_t)F;
    std::vector<Analysis> an(F);
#pragma omp parallel for num_threads(omp) schedule(dynamic, 1)
    for (int64_t f = 0; f < (int64_t)F; ++f) an[f] = analyze_feature(x + f * n, n, cfg, user_cat[f]);
    // compute_groups (feature_analysis.rs:655-751) + create_bundle_plan filter (bundling.rs:395-400):
    // sparse storage and EFB bundles are outside this restatement.
    for (uint64_t f = 0; f < F; ++f) {
        if (an[f].is_trivial) continue;
        bool bundle_candidate = !an[f].is_numeric && an[f].density <= 1.0 - (double)cfg.sparsity_threshold;
        if (an[f].is_sparse || (cfg.enable_bundling && bundle_candidate)) {
            g_err = "feature " + std::to_string(f) + " would use sparse storage; not supported";
            return BST_ERR_UNSUPPORTED;
        }
    }
    // create_bin_mappers (dataset.rs:592-681)
    std::vector<uint32_t> sidx = sample_indices(n, cfg.binning_sample_cnt);
    b.mappers.resize(F);
#pragma omp parallel for num_threads(omp) schedule(dynamic, 1)
    for (int64_t f = 0; f < (int64_t)F; ++f) {
        const float* col = x + f * n;
        bool has_nan = an[f].n_nan > 0;
        if (an[f].is_numeric) {
            std::vector<float> vals;
            if (sidx.empty())
                vals.assign(col, col + n);
            else {
                vals.resize(sidx.size());
                for (size_t i = 0; i < sidx.size(); ++i) vals[i] = col[sidx[i]];
            }
            b.mappers[f] = bin_numeric(vals, cfg.max_bins, has_nan);
        } else {
            std::unordered_set<int32_t> seen;
            for (uint64_t i = 0; i < n; ++i)
                if (std::isfinite(col[i])) seen.insert(sat_i32(col[i]));
            std::vector<int32_t> cats(seen.begin(), seen.end());
            std::sort(cats.begin(), cats.end());
            if (cats.empty()) cats.push_back(0);
            b.mappers[f] = BinMapper::categorical_from(std::move(cats), MISSING_NONE, 0);
        }
    }
    // feature_views (dataset.rs:460-524): standalone non-trivial features in order.
    uint32_t off = 0;
    for (uint64_t f = 0; f < F; ++f) {
        if (an[f].is_trivial) continue;
        const BinMapper& m = b.mappers[f];
        b.col_feature.push_back((uint32_t)f);
        b.col_nbins.push_back(m.n_bins);
        b.col_cat.push_back(m.categorical ? 1 : 0);
        b.col_missing.push_back(m.missing != MISSING_NONE ? 1 : 0);
        b.col_default.push_back(m.default_bin);
        b.col_offset.push_back(off);
        off += m.n_bins;
    }
    b.total_bins = off;
    // build_numeric_dense / build_categorical_dense (dataset.rs:782-842)
    const int64_t n_cols = (int64_t)b.col_feature.size();
    b.col_bins.resize(n_cols);
#pragma omp parallel for num_threads(omp) schedule(dynamic, 1)
    for (int64_t c = 0; c < n_cols; ++c) {
        const uint32_t f = b.col_feature[c];
        const BinMapper& m = b.mappers[f];
        std::vector<uint16_t> bins(n);
        const float* col = x + (uint64_t)f * n;
        for (uint64_t i = 0; i < n; ++i) bins[i] = (uint16_t)m.value_to_bin((double)col[i]);
        b.col_bins[c] = std::move(bins);
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Objectives (training/objectives/*)
// ---------------------------------------------------------------------------

namespace {

inline float w_at(const float* w, uint64_t i) { return w ? w[i] : 1.0f; }

}  // namespace

// f32 exp as the correctly rounded value: glibc's f64 exp rounded once to
// f32. The reference calls the platform's expf (f32::exp); glibc's expf has a
// 0.502 ULP bound, so the two can differ in the last bit for rare inputs, and
// the reference's own tests compare exp-derived values with tolerances.
inline float exp_f32(float x) { return (float)std::exp((double)x); }

namespace {

// Objective parameters: the pinball alphas (one output each) and the
// pseudo-Huber delta.
struct ObjP {
    const float* alpha = nullptr;
    uint32_t n_alpha = 0;
    float delta = 1.0f;
    static ObjP of(const bst_config& c) {
        ObjP p;
        p.alpha = c.quantile_alpha;
        p.n_alpha = c.n_quantiles;
        p.delta = c.huber_delta;
        return p;
    }
    float alpha_at(uint32_t o) const { return alpha && o < n_alpha ? alpha[o] : 0.5f; }
};

// f32::signum: +-1 with the sign bit (so +-0 give +-1), NaN for NaN.
inline float signum_f32(float v) { return std::isnan(v) ? v : std::copysign(1.0f, v); }

// regression.rs:20-43, 80-104, 129-155, 183-215, 243-271; classification.rs:19-52, 88-117, 141-187
void gradients(int obj, const ObjP& op, uint32_t G, const float* preds, const float* y, const float* w, uint64_t n,
               float* grad, float* hess) {
    const float HESS_MIN = 1e-6f;
    if (obj == BST_OBJ_ABSOLUTE || obj == BST_OBJ_PINBALL || obj == BST_OBJ_PSEUDO_HUBER || obj == BST_OBJ_POISSON ||
        obj == BST_OBJ_HINGE) {
        const float inv_delta_sq = 1.0f / (op.delta * op.delta);
        for (uint32_t o = 0; o < G; ++o) {
            const float alpha = op.alpha_at(o);
            for (uint64_t i = 0; i < n; ++i) {
                const float wi = w_at(w, i), p = preds[o * n + i], t = y[i];
                float g, h;
                if (obj == BST_OBJ_ABSOLUTE) {
                    g = wi * signum_f32(p - t);
                    h = wi;
                } else if (obj == BST_OBJ_PINBALL) {
                    g = wi * ((p - t) < 0.0f ? -alpha : 1.0f - alpha);
                    h = wi;
                } else if (obj == BST_OBJ_PSEUDO_HUBER) {
                    const float r = p - t, r_sq = r * r;
                    const float factor = 1.0f + r_sq * inv_delta_sq, sq = std::sqrt(factor);
                    g = wi * r / sq;
                    h = wi / (factor * sq);
                } else if (obj == BST_OBJ_POISSON) {
                    const float pc = p < -30.0f ? -30.0f : (p > 30.0f ? 30.0f : p);
                    const float e = exp_f32(pc);
                    g = wi * (e - t);
                    h = std::fmax(wi * e, HESS_MIN);
                } else {  // hinge: labels {0, 1} as {-1, +1}
                    const float yy = t > 0.5f ? 1.0f : -1.0f, margin = yy * p;
                    g = margin < 1.0f ? -wi * yy : 0.0f;
                    h = wi;
                }
                grad[o * n + i] = g;
                hess[o * n + i] = h;
            }
        }
        return;
    }
    if (obj == BST_OBJ_SQUARED) {
        for (uint32_t o = 0; o < G; ++o)
            for (uint64_t i = 0; i < n; ++i) {
                float wi = w_at(w, i);
                grad[o * n + i] = wi * (preds[o * n + i] - y[i]);
                hess[o * n + i] = wi;
            }
    } else if (obj == BST_OBJ_LOGISTIC) {
        for (uint32_t o = 0; o < G; ++o)
            for (uint64_t i = 0; i < n; ++i) {
                float wi = w_at(w, i);
                float p = 1.0f / (1.0f + exp_f32(-preds[o * n + i]));
                grad[o * n + i] = wi * (p - y[i]);
                hess[o * n + i] = std::fmax(wi * p * (1.0f - p), HESS_MIN);
            }
    } else {  // softmax
        for (uint64_t i = 0; i < n; ++i) {
            float wi = w_at(w, i);
            uint64_t label = sat_usize(y[i]);
            float mx = -std::numeric_limits<float>::infinity();
            for (uint32_t c = 0; c < G; ++c) mx = std::fmax(mx, preds[c * n + i]);
            float sum = -0.0f;
            for (uint32_t c = 0; c < G; ++c) sum += exp_f32(preds[c * n + i] - mx);
            for (uint32_t c = 0; c < G; ++c) {
                float p = exp_f32(preds[c * n + i] - mx) / sum;
                float ind = (c == label) ? 1.0f : 0.0f;
                grad[c * n + i] = wi * (p - ind);
                hess[c * n + i] = std::fmax(wi * p * (1.0f - p), HESS_MIN);
            }
        }
    }
}

inline double clamp64(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

// compute_weighted_quantile (regression.rs:307-333): (value, weight) pairs
// sorted stably by value; the first value whose f32 running weight reaches
// alpha x the f32 total of the sorted weights.
float weighted_quantile_base(const float* y, const float* w, uint64_t n, float alpha) {
    if (n == 0) return 0.0f;
    std::vector<std::pair<float, float>> v(n);
    for (uint64_t i = 0; i < n; ++i) v[i] = {y[i], w_at(w, i)};
    std::stable_sort(v.begin(), v.end(), [](const std::pair<float, float>& a, const std::pair<float, float>& b) {
        return a.first < b.first;
    });
    float total = 0.0f;
    for (const auto& e : v) total += e.second;
    const float target = alpha * total;
    float cum = 0.0f;
    for (const auto& e : v) {
        cum += e.second;
        if (cum >= target) return e.first;
    }
    return v.back().first;
}

// unweighted_quantile_indexed (utils.rs:17-53): the element of rank
// ceil(alpha n) - 1 (clamped to [0, n - 1]) by value.
float unweighted_quantile(std::vector<float> v, float alpha) {
    const size_t n = v.size();
    if (n == 0) return std::numeric_limits<float>::quiet_NaN();
    if (n == 1) return v[0];
    const float c = std::ceil(alpha * (float)n);
    size_t k = c > 0.0f ? (size_t)c : 0;
    k = k > 0 ? k - 1 : 0;
    k = std::min(k, n - 1);
    std::nth_element(v.begin(), v.begin() + k, v.end());
    return v[k];
}

// weighted_quantile_indexed (utils.rs:81-135): values sorted stably, the
// f32 total of the weights in the given order, the first value whose f32
// running weight reaches alpha x total.
float weighted_quantile(const std::vector<float>& v, const std::vector<float>& wt, float alpha) {
    const size_t n = v.size();
    if (n == 0) return std::numeric_limits<float>::quiet_NaN();
    if (n == 1) return v[0];
    std::vector<uint32_t> ord(n);
    for (size_t i = 0; i < n; ++i) ord[i] = (uint32_t)i;
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return v[a] < v[b]; });
    float total = 0.0f;
    for (size_t i = 0; i < n; ++i) total += wt[i];
    const float threshold = total * alpha;
    float cum = 0.0f;
    for (uint32_t i : ord) {
        cum += wt[i];
        if (cum >= threshold) return v[i];
    }
    return v[ord[n - 1]];
}

// regression.rs:45-69, 106-118, 157-173, 217-228, 273-298; classification.rs:54-76, 119-125, 189-222
void base_score(int obj, const ObjP& op, uint32_t G, const float* y, const float* w, uint64_t n, float* out) {
    if (n == 0) {
        for (uint32_t g = 0; g < G; ++g) out[g] = 0.0f;
        return;
    }
    if (obj == BST_OBJ_ABSOLUTE || obj == BST_OBJ_PSEUDO_HUBER) {
        out[0] = weighted_quantile_base(y, w, n, 0.5f);
        return;
    }
    if (obj == BST_OBJ_PINBALL) {
        for (uint32_t g = 0; g < G; ++g) out[g] = weighted_quantile_base(y, w, n, op.alpha_at(g));
        return;
    }
    if (obj == BST_OBJ_HINGE) {
        out[0] = 0.0f;
        return;
    }
    if (obj == BST_OBJ_POISSON) {
        double sw = 0, swy = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const double wi = (double)w_at(w, i);
            sw = sw + wi;
            swy = swy + wi * (double)y[i];
        }
        const double mean = sw > 0.0 ? std::fmax(swy / sw, 1e-7) : 1.0;
        out[0] = f64_to_f32(std::log(mean));
        return;
    }
    if (obj == BST_OBJ_SQUARED) {
        double sw = 0, swy = 0;
        for (uint64_t i = 0; i < n; ++i) {
            double wi = (double)w_at(w, i);
            sw = sw + wi;
            swy = swy + wi * (double)y[i];
        }
        out[0] = sw > 0.0 ? f64_to_f32(swy / sw) : 0.0f;
    } else if (obj == BST_OBJ_LOGISTIC) {
        double pos = 0, tot = 0;
        for (uint64_t i = 0; i < n; ++i) {
            double wi = (double)w_at(w, i);
            pos = pos + wi * (double)y[i];
            tot = tot + wi;
        }
        double p = clamp64(pos / tot, 1e-7, 1.0 - 1e-7);
        out[0] = f64_to_f32(std::log(p / (1.0 - p)));
    } else {
        std::vector<double> cw(G, 0.0);
        double tot = 0;
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t label = sat_usize(y[i]);
            double wi = (double)w_at(w, i);
            if (label < G) cw[label] += wi;
            tot += wi;
        }
        for (uint32_t g = 0; g < G; ++g) out[g] = f64_to_f32(std::log(clamp64(cw[g] / tot, 1e-7, 1.0 - 1e-7)));
    }
}

// ---------------------------------------------------------------------------
// Gain (training/gbdt/split/gain.rs)
// ---------------------------------------------------------------------------

struct GainParams {
    float lambda = 1.0f, alpha = 0.0f, min_gain = 0.0f, min_child_weight = 1.0f;
    uint32_t min_samples_leaf = 1;
    // Units of the histogram sums: 1.0 for f32 gradients; the quantisation
    // steps when the histograms hold exact integer sums of quantised values
    // (every prefix / difference stays an exact integer, converted at use).
    double sg = 1.0, sh = 1.0;
};

struct NodeGainContext {  // gain.rs:16-52
    double lambda, gain_offset;
    NodeGainContext(double pg, double ph, const GainParams& p) {
        lambda = (double)p.lambda;
        double parent_score = pg * pg / (ph + lambda);
        gain_offset = 0.5 * parent_score + (double)p.min_gain;
    }
    float gain(double gl, double hl, double gr, double hr) const {
        double sl = gl * gl / (hl + lambda);
        double sr = gr * gr / (hr + lambda);
        return f64_to_f32(0.5 * (sl + sr) - gain_offset);
    }
};

inline bool is_valid_split(const GainParams& p, double hl, double hr, uint32_t cl, uint32_t cr) {
    double mw = (double)p.min_child_weight;
    return hl >= mw && hr >= mw && cl >= p.min_samples_leaf && cr >= p.min_samples_leaf;
}

float leaf_weight(const GainParams& p, double g, double h) {  // gain.rs:151-168
    double lambda = (double)p.lambda, alpha = (double)p.alpha;
    if (alpha == 0.0) return f64_to_f32(-g / (h + lambda));
    double ag = std::fabs(g);
    if (ag <= alpha) return 0.0f;
    double sign = g > 0.0 ? -1.0 : 1.0;
    return f64_to_f32(sign * (ag - alpha) / (h + lambda));
}

inline uint32_t sat_sub(uint32_t a, uint32_t b) { return a > b ? a - b : 0; }

// ---------------------------------------------------------------------------
// Split search (training/gbdt/split/find.rs)
// ---------------------------------------------------------------------------

struct Split {  // split/types.rs:34-102
    uint32_t feature = 0;
    float gain = -std::numeric_limits<float>::infinity();
    bool default_left = false;
    bool categorical = false;
    uint32_t bin = 0;
    std::vector<uint32_t> left_cats;  // sorted ascending
    bool valid() const { return gain > -std::numeric_limits<float>::infinity(); }
};

typedef std::pair<double, double> HBin;

// find.rs:286-407
Split find_numerical(const HBin* bins, uint32_t n_bins, uint32_t feature, double pg, double ph,
                     uint32_t pc, bool has_missing, const GainParams& gp,
                     const NodeGainContext& ctx) {
    Split best;
    if (n_bins < 2) return best;
    double lg = 0.0, lh = 0.0;
    uint32_t lc = 0;
    for (uint32_t bin = 0; bin < n_bins - 1; ++bin) {
        lg += bins[bin].first;
        lh += bins[bin].second;
        lc += 1;
        double rg = pg - lg, rh = ph - lh;
        uint32_t rc = sat_sub(pc, lc);
        if (is_valid_split(gp, lh * gp.sh, rh * gp.sh, lc, rc)) {
            float g = ctx.gain(lg * gp.sg, lh * gp.sh, rg * gp.sg, rh * gp.sh);
            if (g > best.gain) {
                best.feature = feature;
                best.gain = g;
                best.default_left = false;
                best.categorical = false;
                best.bin = bin;
            }
        }
    }
    if (has_missing) {
        double rg = 0.0, rh = 0.0;
        uint32_t rc = 0;
        uint32_t max_excl = n_bins - 1;  // missing bin is last
        for (uint32_t bin = max_excl; bin-- > 1;) {
            rg += bins[bin].first;
            rh += bins[bin].second;
            rc += 1;
            double lg2 = pg - rg, lh2 = ph - rh;
            uint32_t lc2 = sat_sub(pc, rc);
            if (is_valid_split(gp, lh2 * gp.sh, rh * gp.sh, lc2, rc)) {
                float g = ctx.gain(lg2 * gp.sg, lh2 * gp.sh, rg * gp.sg, rh * gp.sh);
                if (g > best.gain) {
                    best.feature = feature;
                    best.gain = g;
                    best.default_left = true;
                    best.categorical = false;
                    best.bin = bin - 1;
                }
            }
        }
    }
    return best;
}

// find.rs:472-508
Split find_onehot(const HBin* bins, uint32_t n_cats, uint32_t feature, double pg, double ph,
                  uint32_t pc, const GainParams& gp, const NodeGainContext& ctx) {
    Split best;
    for (uint32_t c = 0; c < n_cats; ++c) {
        double lg = bins[c].first, lh = bins[c].second;
        uint32_t lc = 1;
        double rg = pg - lg, rh = ph - lh;
        uint32_t rc = sat_sub(pc, lc);
        if (is_valid_split(gp, lh * gp.sh, rh * gp.sh, lc, rc)) {
            float g = ctx.gain(lg * gp.sg, lh * gp.sh, rg * gp.sg, rh * gp.sh);
            if (g > best.gain) {
                best.feature = feature;
                best.gain = g;
                best.default_left = false;
                best.categorical = true;
                best.left_cats = {c};
            }
        }
    }
    return best;
}

// find.rs:511-573 (and the identical find_sorted_split_with_scratch :583-644)
Split find_sorted(const HBin* bins, uint32_t n_cats, uint32_t feature, double pg, double ph,
                  uint32_t pc, const GainParams& gp, const NodeGainContext& ctx) {
    Split best;
    std::vector<std::pair<uint32_t, double>> s;
    for (uint32_t c = 0; c < n_cats; ++c) {
        const double gg = bins[c].first * gp.sg, hh = bins[c].second * gp.sh;
        if (hh > 1e-10) s.push_back({c, -gg / (hh + 1e-6)});
    }
    if (s.size() < 2) return best;
    std::stable_sort(s.begin(), s.end(),
                     [](const std::pair<uint32_t, double>& a, const std::pair<uint32_t, double>& b) {
                         return a.second < b.second;
                     });
    std::vector<uint32_t> left;
    double lg = 0.0, lh = 0.0;
    uint32_t lc = 0;
    for (size_t i = 0; i + 1 < s.size(); ++i) {
        uint32_t c = s[i].first;
        left.push_back(c);
        lg += bins[c].first;
        lh += bins[c].second;
        lc += 1;
        double rg = pg - lg, rh = ph - lh;
        uint32_t rc = sat_sub(pc, lc);
        if (is_valid_split(gp, lh * gp.sh, rh * gp.sh, lc, rc)) {
            float g = ctx.gain(lg * gp.sg, lh * gp.sh, rg * gp.sg, rh * gp.sh);
            if (g > best.gain) {
                best.feature = feature;
                best.gain = g;
                best.default_left = false;
                best.categorical = true;
                best.left_cats = left;
                std::sort(best.left_cats.begin(), best.left_cats.end());
            }
        }
    }
    return best;
}

struct SplitterCfg {
    GainParams gp;
    uint32_t max_onehot_cats = 4;
    bool parallel = false;  // rayon reduction order (find.rs:219-270)
    int omp_threads = 1;
};

// find.rs:113-270
// feats (or null): the node's searched columns in ascending order (column
// sampling), n_sel of them; null: all n_feat.
Split find_split(const HBin* hist, const uint32_t* offs, const uint32_t* nb, const uint8_t* is_cat,
                 const uint8_t* has_missing, uint32_t n_feat, double pg, double ph, uint32_t pc,
                 const SplitterCfg& sc, const uint32_t* feats = nullptr, uint32_t n_sel = 0) {
    NodeGainContext ctx(pg * sc.gp.sg, ph * sc.gp.sh, sc.gp);
    const uint32_t n_search = feats ? n_sel : n_feat;
    bool par = sc.parallel && n_search >= 16;  // MIN_FEATURES_PARALLEL over the searched features (find.rs:18,125)
    std::vector<Split> per(n_feat);
    auto eval = [&](uint32_t f) {
        const HBin* bins = hist + offs[f];
        if (is_cat[f]) {
            if (nb[f] < 2)
                per[f] = Split();
            else if (nb[f] <= sc.max_onehot_cats)
                per[f] = find_onehot(bins, nb[f], f, pg, ph, pc, sc.gp, ctx);
            else
                per[f] = find_sorted(bins, nb[f], f, pg, ph, pc, sc.gp, ctx);
        } else {
            per[f] = find_numerical(bins, nb[f], f, pg, ph, pc, has_missing[f] != 0, sc.gp, ctx);
        }
    };
#ifdef _OPENMP
    if (sc.omp_threads > 1 && n_search >= 16) {
#pragma omp parallel for num_threads(sc.omp_threads) schedule(dynamic, 4)
        for (int64_t i = 0; i < (int64_t)n_search; ++i) eval(feats ? feats[i] : (uint32_t)i);
    } else
#endif
        for (uint32_t i = 0; i < n_search; ++i) eval(feats ? feats[i] : i);
    Split best;
    for (uint32_t i = 0; i < n_search; ++i) {
        const uint32_t f = feats ? feats[i] : i;
        if (par) {
            // reduce(|a, b| if a.gain > b.gain { a } else { b }): ties go to the later item
            if (!(best.gain > per[f].gain)) best = per[f];
        } else {
            if (per[f].gain > best.gain) best = per[f];
        }
    }
    return best;
}

// ---------------------------------------------------------------------------
// Histogram pool (training/gbdt/histograms/pool.rs:83-499), exact port
// ---------------------------------------------------------------------------

struct HistogramPool {
    std::vector<HBin> data;
    size_t total_bins = 0, cache_size = 0, total_nodes = 0;
    std::vector<int32_t> node_to_slot, slot_to_node;
    std::vector<uint64_t> last_used;
    uint64_t current_time = 0;
    bool identity = false;
    uint64_t epoch = 1;
    std::vector<uint64_t> slot_epoch;
    std::vector<uint8_t> pinned;

    void init(size_t tb, size_t cache, size_t nodes) {
        cache = std::max<size_t>(cache, 2);  // grower.rs:144 cache_size.max(2)
        total_bins = tb;
        cache_size = std::min(cache, nodes);
        total_nodes = nodes;
        identity = cache_size >= total_nodes;
        data.assign(cache_size * total_bins, HBin(0.0, 0.0));
        if (identity) {
            slot_epoch.assign(cache_size, 0);
        } else {
            node_to_slot.assign(total_nodes, -1);
            slot_to_node.assign(cache_size, -1);
            last_used.assign(cache_size, 0);
            pinned.assign(cache_size, 0);
        }
        current_time = 0;
        epoch = 1;
    }
    void reset_mappings() {
        if (identity) {
            epoch += 1;
            if (epoch == 0) epoch = 1;
            return;
        }
        current_time = 0;
        std::fill(node_to_slot.begin(), node_to_slot.end(), -1);
        std::fill(slot_to_node.begin(), slot_to_node.end(), -1);
        std::fill(last_used.begin(), last_used.end(), 0);
        std::fill(pinned.begin(), pinned.end(), 0);
    }
    int resolve(uint32_t node) const {
        if (identity) {
            if (node >= cache_size) return -1;
            return slot_epoch[node] == epoch ? (int)node : -1;
        }
        return node_to_slot[node];
    }
    void pin(uint32_t node) {
        if (identity) return;
        int s = resolve(node);
        if (s >= 0) pinned[s] = 1;
    }
    void unpin(uint32_t node) {
        if (identity) return;
        int s = resolve(node);
        if (s >= 0) pinned[s] = 0;
    }
    size_t find_lru() const {
        uint64_t mn = UINT64_MAX;
        size_t slot = 0;
        bool found = false;
        for (size_t s = 0; s < cache_size; ++s) {
            if (pinned[s]) continue;
            if (last_used[s] < mn) {
                mn = last_used[s];
                slot = s;
                found = true;
            }
        }
        (void)found;
        return slot;
    }
    // returns slot, sets hit
    size_t acquire(uint32_t node, bool& hit) {
        if (identity) {
            if (slot_epoch[node] == epoch) {
                hit = true;
                return node;
            }
            slot_epoch[node] = epoch;
            hit = false;
            return node;
        }
        int ex = node_to_slot[node];
        if (ex >= 0) {
            current_time += 1;
            last_used[ex] = current_time;
            hit = true;
            return (size_t)ex;
        }
        size_t s = find_lru();
        current_time += 1;
        last_used[s] = current_time;
        int prev = slot_to_node[s];
        if (prev >= 0) node_to_slot[prev] = -1;
        node_to_slot[node] = (int32_t)s;
        slot_to_node[s] = (int32_t)node;
        hit = false;
        return s;
    }
    void release(uint32_t node) {
        if (identity) return;
        int s = node_to_slot[node];
        if (s >= 0) {
            node_to_slot[node] = -1;
            slot_to_node[s] = -1;
            last_used[s] = 0;
            pinned[s] = 0;
        }
    }
    void move_mapping(uint32_t from, uint32_t to) {
        if (identity) {
            if (from == to) return;
            std::copy(data.begin() + from * total_bins, data.begin() + (from + 1) * total_bins,
                      data.begin() + to * total_bins);
            if (from < cache_size && to < cache_size) {
                slot_epoch[to] = epoch;
                slot_epoch[from] = 0;
            }
            return;
        }
        int s = node_to_slot[from];
        if (s < 0) return;
        node_to_slot[from] = -1;
        node_to_slot[to] = s;
        slot_to_node[s] = (int32_t)to;
        current_time += 1;
        last_used[s] = current_time;
    }
    HBin* slot_ptr(size_t s) { return data.data() + s * total_bins; }
    void subtract(uint32_t target, uint32_t source) {
        HBin* t = slot_ptr(resolve(target));
        HBin* s = slot_ptr(resolve(source));
        for (size_t i = 0; i < total_bins; ++i) {
            t[i].first -= s[i].first;
            t[i].second -= s[i].second;
        }
    }
};

// ---------------------------------------------------------------------------
// Row partitioner (training/gbdt/partition.rs:55-382)
// ---------------------------------------------------------------------------

struct RowPartitioner {
    std::vector<uint32_t> indices, scratch, begin, count;
    uint32_t n_leaves = 0;
    void init(uint64_t n, size_t max_leaves) {
        indices.resize(n);
        scratch.assign(n, 0);
        begin.assign(max_leaves, 0);
        count.assign(max_leaves, 0);
    }
    void reset(uint64_t n) {
        for (uint64_t i = 0; i < n; ++i) indices[i] = (uint32_t)i;
        std::fill(begin.begin(), begin.end(), 0);
        std::fill(count.begin(), count.end(), 0);
        count[0] = (uint32_t)n;
        n_leaves = 1;
    }
    // stable_partition_range (partition.rs:73-145) + split (:296-382)
    template <class F>
    uint32_t split(uint32_t leaf, F goes_left, uint32_t& lc, uint32_t& rc) {
        size_t b = begin[leaf], c = count[leaf], e = b + c;
        size_t lw = b, rw = e;
        for (size_t i = b; i < e; ++i) {
            uint32_t idx = indices[i];
            if (goes_left(idx))
                scratch[lw++] = idx;
            else
                scratch[--rw] = idx;
        }
        std::reverse(scratch.begin() + lw, scratch.begin() + e);
        std::copy(scratch.begin() + b, scratch.begin() + e, indices.begin() + b);
        lc = (uint32_t)(lw - b);
        rc = (uint32_t)(c - lc);
        count[leaf] = lc;
        uint32_t right = n_leaves++;
        begin[right] = (uint32_t)(b + lc);
        count[right] = rc;
        return right;
    }
};

// ---------------------------------------------------------------------------
// Trees (repr/gbdt/mutable_tree.rs, tree.rs, categories.rs)
// ---------------------------------------------------------------------------

struct Tree {
    std::vector<uint32_t> split_index, left, right;
    std::vector<float> threshold, leaf, gain, cover;
    std::vector<uint8_t> default_left, is_leaf, split_type;
    std::vector<std::pair<uint32_t, std::vector<uint32_t>>> cat_nodes;  // (node, bitset words)
    // frozen categories (categories.rs:29-117)
    std::vector<uint32_t> seg_start, seg_size, cat_words;
    // training detail
    std::vector<uint32_t> split_bin;
    std::vector<double> grad_sum, hess_sum;
    std::vector<uint32_t> row_leaf;
    uint32_t group = 0;

    uint32_t alloc() {
        split_index.push_back(0);
        threshold.push_back(0.0f);
        left.push_back(0);
        right.push_back(0);
        default_left.push_back(0);
        is_leaf.push_back(0);
        leaf.push_back(0.0f);
        split_type.push_back(0);
        gain.push_back(0.0f);
        cover.push_back(0.0f);
        split_bin.push_back(0xFFFFFFFFu);
        grad_sum.push_back(0.0);
        hess_sum.push_back(0.0);
        return (uint32_t)split_index.size() - 1;
    }
    void freeze() {  // mutable_tree.rs:299-335
        size_t nn = split_index.size();
        seg_start.assign(nn, 0);
        seg_size.assign(nn, 0);
        cat_words.clear();
        std::sort(cat_nodes.begin(), cat_nodes.end(),
                  [](const std::pair<uint32_t, std::vector<uint32_t>>& a,
                     const std::pair<uint32_t, std::vector<uint32_t>>& b) { return a.first < b.first; });
        for (auto& cn : cat_nodes) {
            seg_start[cn.first] = (uint32_t)cat_words.size();
            seg_size[cn.first] = (uint32_t)cn.second.size();
            cat_words.insert(cat_words.end(), cn.second.begin(), cn.second.end());
        }
    }
    bool goes_right(uint32_t node, uint32_t cat) const {  // categories.rs:76-91
        uint32_t sz = seg_size[node];
        if (sz == 0) return false;
        uint32_t wi = cat >> 5, bi = cat & 31;
        if (wi >= sz) return false;
        return (cat_words[seg_start[node] + wi] >> bi) & 1u;
    }
    // tree_view.rs:119-160 traverse_to_leaf_from
    uint32_t traverse(const float* x, uint64_t stride) const {
        uint32_t node = 0;
        while (!is_leaf[node]) {
            float v = x[(uint64_t)split_index[node] * stride];
            if (std::isnan(v))
                node = default_left[node] ? left[node] : right[node];
            else if (split_type[node] == 0)
                node = v < threshold[node] ? left[node] : right[node];
            else
                node = goes_right(node, sat_u32(v)) ? right[node] : left[node];
        }
        return node;
    }
};

// categories.rs:145-161
std::vector<uint32_t> categories_to_bitset(const std::vector<uint32_t>& cats) {
    if (cats.empty()) return {};
    uint32_t mx = *std::max_element(cats.begin(), cats.end());
    std::vector<uint32_t> bs((mx >> 5) + 1, 0);
    for (uint32_t c : cats) bs[c >> 5] |= 1u << (c & 31);
    return bs;
}

// ---------------------------------------------------------------------------
// Tree grower (training/gbdt/grower.rs:105-752, expansion.rs)
// ---------------------------------------------------------------------------

struct Candidate {  // expansion.rs:246-300
    uint32_t node, tree_node;
    uint32_t depth;
    Split split;
    double g, h;
    uint32_t count;
};

struct TrainCfg {
    SplitterCfg sc;
    float learning_rate = 0.3f;
    bool leafwise = false;
    uint32_t max_depth = 6, max_leaves = 31;
    size_t cache_size = 8;
    float colsample_bytree = 1.0f, colsample_bylevel = 1.0f;
    uint64_t seed = 42;
};

// ---------------------------------------------------------------------------
// Column sampling (training/sampling/column.rs): the reference seeds it from
// OS entropy (grower.rs:150-151, column.rs:137-142), so its draws are not
// reproducible; the engine and this restatement draw from a splitmix64
// stream keyed by (seed, round, output, depth) and apply the reference's
// rule: ceil(n * colsample_bytree) columns per tree, ceil(|tree| *
// colsample_bylevel) of those per depth, by a partial Fisher-Yates shuffle
// (sample_k_inplace, column.rs:266-283), in ascending order.
// ---------------------------------------------------------------------------
static uint64_t cs_mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
struct ColRng {
    uint64_t s;
    ColRng(uint64_t seed, uint32_t round, uint32_t output, uint32_t depth) {
        s = cs_mix(seed ^ (0x9E3779B97F4A7C15ull * (1ull + round)));
        s = cs_mix(s ^ (0xC2B2AE3D27D4EB4Full * (1ull + output)));
        s = cs_mix(s ^ (0x165667B19E3779F9ull * (1ull + depth)));
    }
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ull;
        return cs_mix(s);
    }
};
static bool cs_active(float rate) { return std::fabs(rate - 1.0f) >= 1e-6f; }

// Uniform row sampling (training/sampling/row.rs:168-210) with the
// reference's generator: rand 0.8 SmallRng = Xoshiro256++ seeded by four
// SplitMix64 outputs (seed_from_u64), gen_range(0..=i) by
// UniformInt::sample_single_inclusive (128-bit multiply, zone rejection),
// reservoir sampling of k = max(1, trunc(f32(n) * rate)) rows.
struct OracleRowSampler {
    uint64_t s[4];
    explicit OracleRowSampler(uint64_t seed) {
        for (int i = 0; i < 4; ++i) {
            seed += 0x9E3779B97F4A7C15ull;
            s[i] = cs_mix(seed);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[0] + s[3], 23) + s[0];
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    uint64_t gen_range_inclusive(uint64_t high) {
        const uint64_t range = high + 1;
        const uint64_t zone = (range << __builtin_clzll(range)) - 1;
        for (;;) {
            const unsigned __int128 m = (unsigned __int128)next() * range;
            if ((uint64_t)m <= zone) return (uint64_t)(m >> 64);
        }
    }
    uint64_t sample(uint64_t n, float rate, std::vector<uint8_t>& mask) {
        uint64_t k = (uint64_t)((float)n * rate);
        k = std::min<uint64_t>(std::max<uint64_t>(k, 1), n);
        std::vector<uint32_t> idx(k);
        for (uint64_t i = 0; i < k; ++i) idx[i] = (uint32_t)i;
        for (uint64_t i = k; i < n; ++i) {
            const uint64_t j = gen_range_inclusive(i);
            if (j < k) idx[j] = (uint32_t)i;
        }
        mask.assign(n, 0);
        for (uint32_t r : idx) mask[r] = 1;
        return k;
    }
    // rng.gen::<f32>() of rand 0.8: the top 24 bits of next_u32 (the upper
    // half of a Xoshiro256++ output) times 2^-24
    float gen_f32() {
        const uint32_t u = (uint32_t)(next() >> 32);
        return (float)(u >> 8) * (1.0f / 16777216.0f);
    }
    // sample_goss (row.rs:214-280) on one output's grad / hess (scaled in
    // place for the sampled small-gradient rows); mask: 1 kept, 0 left out
    uint64_t goss(float* g, float* h, uint64_t n, float top_rate, float other_rate, std::vector<uint8_t>& mask) {
        std::vector<float> mag(n);
        for (uint64_t i = 0; i < n; ++i) mag[i] = std::fabs(g[i] * h[i]);
        uint64_t top_k = (uint64_t)((float)n * top_rate);
        top_k = std::min<uint64_t>(std::max<uint64_t>(top_k, 1), n - 1);
        uint64_t other_k = std::max<uint64_t>((uint64_t)((float)n * other_rate), 1);
        std::vector<float> sorted(mag);
        std::nth_element(sorted.begin(), sorted.begin() + (n - top_k), sorted.end());
        const float threshold = sorted[n - top_k];
        const float multiply = (float)(n - top_k) / (float)other_k;
        uint64_t big = 0, small = 0;
        mask.assign(n, 0);
        for (uint64_t i = 0; i < n; ++i) {
            if (mag[i] >= threshold) {
                mask[i] = 1;
                ++big;
                continue;
            }
            const uint64_t need = other_k > small ? other_k - small : 0;
            const uint64_t top_left = top_k > big ? top_k - big : 0;
            const uint64_t rest = (n - i) > top_left ? (n - i) - top_left : 0;
            if (rest > 0) {
                const float prob = (float)need / (float)rest;
                if (gen_f32() < prob) {
                    mask[i] = 1;
                    ++small;
                    g[i] *= multiply;
                    h[i] *= multiply;
                }
            }
        }
        return big + small;
    }
};
static void cs_sample(std::vector<uint32_t>& v, float rate, ColRng rng) {
    const size_t n = v.size();
    size_t k = (size_t)std::ceil((float)n * rate);
    k = std::min(std::max<size_t>(k, 1), n);
    if (k >= n) return;
    for (size_t i = 0; i < k; ++i) std::swap(v[i], v[rng.next() % (n - i) + i]);
    v.resize(k);
    std::sort(v.begin(), v.end());
}

struct Grower {
    const orc_binned* ds;
    TrainCfg tc;
    HistogramPool pool;
    RowPartitioner part;
    std::vector<float> last_leaf;  // by partitioner node
    std::vector<std::pair<uint32_t, uint32_t>> leaf_map;
    std::vector<std::pair<float, float>> ordered;
    Tree tree;
    const float* grad = nullptr;
    const float* hess = nullptr;
    // Quantised training: grad/hess above are the quantised integers (as
    // floats), histogram sums are exact integers, and leaves are solved from
    // the f32 gradients rgrad/rhess summed in f64 over the leaf's rows.
    const float* rgrad = nullptr;
    const float* rhess = nullptr;

    void init(const orc_binned* b, const TrainCfg& cfg) {
        ds = b;
        tc = cfg;
        uint32_t max_leaves = tc.leafwise ? tc.max_leaves : (1u << tc.max_depth);
        size_t max_nodes = std::max<size_t>(2 * (size_t)max_leaves >= 1 ? 2 * (size_t)max_leaves - 1 : 0, 63);
        pool.init(b->total_bins, tc.cache_size, max_nodes);
        part.init(b->n, max_nodes);
    }

    // grower.rs:662-730 build_histogram (gathered and contiguous paths both sum in row order)
    void build_histogram(uint32_t node) {
        bool hit;
        size_t slot = pool.acquire(node, hit);
        HBin* h = pool.slot_ptr(slot);
        if (!hit) std::fill(h, h + pool.total_bins, HBin(0.0, 0.0));
        uint32_t b = part.begin[node], c = part.count[node];
        if (c == 0) return;
        const uint32_t* rows = part.indices.data() + b;
        ordered.resize(c);
        for (uint32_t i = 0; i < c; ++i) ordered[i] = {grad[rows[i]], hess[rows[i]]};
        uint32_t nf = (uint32_t)ds->col_feature.size();
        auto one = [&](uint32_t f) {
            HBin* hf = h + ds->col_offset[f];
            const uint16_t* bins = ds->col_bins[f].data();
            for (uint32_t i = 0; i < c; ++i) {
                HBin& s = hf[bins[rows[i]]];
                s.first += (double)ordered[i].first;
                s.second += (double)ordered[i].second;
            }
        };
#ifdef _OPENMP
        // feature-parallel like ops.rs:131-143 (MIN_FEATURES_PARALLEL 4, MIN_WORK 4096)
        if (tc.sc.omp_threads > 1 && nf >= 4 && (uint64_t)c * nf >= 4096) {
#pragma omp parallel for num_threads(tc.sc.omp_threads) schedule(dynamic, 1)
            for (int64_t f = 0; f < (int64_t)nf; ++f) one((uint32_t)f);
        } else
#endif
            for (uint32_t f = 0; f < nf; ++f) one(f);
    }

    std::pair<double, double> sum_gradients(uint32_t node) {  // pool.rs:536-549
        HBin* h = pool.slot_ptr(pool.resolve(node));
        double g = 0.0, hh = 0.0;
        if (ds->col_feature.empty()) return {0.0, 0.0};
        for (uint32_t i = 0; i < ds->col_nbins[0]; ++i) {
            g += h[i].first;
            hh += h[i].second;
        }
        return {g, hh};
    }

    // row sampling: the tree's sampled rows (null: all). The reference's
    // partition holds only the sampled rows (grower.rs:275-276); here every
    // row stays and the others carry zero grad/hess, which adds exact zeros to
    // every f64 sum, while node counts (split validity, smaller child) count
    // the sampled rows as the reference's do.
    const uint8_t* rmask = nullptr;
    uint32_t n_sampled = 0;
    uint32_t sampled_in(uint32_t node) const {
        const uint32_t b = part.begin[node], c = part.count[node];
        if (!rmask) return c;
        uint32_t k = 0;
        for (uint32_t i = 0; i < c; ++i) k += rmask[part.indices[b + i]] != 0;
        return k;
    }

    // column sampling of the tree being grown: its round and output, the
    // tree's columns and each depth's columns (computed on first use)
    uint32_t cs_round = 0, cs_output = 0;
    std::vector<uint32_t> cs_tree;
    std::vector<std::vector<uint32_t>> cs_level;
    void cs_begin_tree() {
        cs_tree.clear();
        cs_level.clear();
        if (!cs_active(tc.colsample_bytree) && !cs_active(tc.colsample_bylevel)) return;
        const uint32_t nc = (uint32_t)ds->col_feature.size();
        for (uint32_t c = 0; c < nc; ++c) cs_tree.push_back(c);
        if (cs_active(tc.colsample_bytree))
            cs_sample(cs_tree, tc.colsample_bytree, ColRng(tc.seed, cs_round, cs_output, 0xFFFFFFFFu));
    }
    const std::vector<uint32_t>* cs_features(uint32_t depth) {
        if (cs_tree.empty()) return nullptr;
        while (cs_level.size() <= depth) {
            std::vector<uint32_t> v = cs_tree;
            if (cs_active(tc.colsample_bylevel))
                cs_sample(v, tc.colsample_bylevel, ColRng(tc.seed, cs_round, cs_output, (uint32_t)cs_level.size()));
            cs_level.push_back(std::move(v));
        }
        return &cs_level[depth];
    }

    Split find(uint32_t node, double g, double h, uint32_t cnt, uint32_t depth) {  // grower.rs:733-752
        int s = pool.resolve(node);
        if (s < 0) return Split();
        const std::vector<uint32_t>* fs = cs_features(depth);
        return find_split(pool.slot_ptr(s), ds->col_offset.data(), ds->col_nbins.data(),
                          ds->col_cat.data(), ds->col_missing.data(),
                          (uint32_t)ds->col_feature.size(), g, h, cnt, tc.sc, fs ? fs->data() : nullptr,
                          fs ? (uint32_t)fs->size() : 0u);
    }

    void record_leaf(uint32_t tree_node, uint32_t pnode, float w) {  // grower.rs:238-250
        if (pnode >= last_leaf.size()) last_leaf.resize(pnode + 1, std::numeric_limits<float>::quiet_NaN());
        last_leaf[pnode] = w * tc.learning_rate;
        leaf_map.push_back({tree_node, pnode});
    }

    // Quantised mode: leaf totals are exact, order-independent sums of the f32
    // gradients on the fixed-point grid 2^-k (k from max|v| and the row count:
    // |round(v 2^k)| <= 2^38 and n 2^k max|v| < 2^62), then scaled back.
    int kg = 0, kh = 0;
    void make_leaf(const Candidate& c) {
        double g = c.g, h = c.h;
        if (rgrad) {
            long long sg = 0, sh = 0;
            const double fg = std::ldexp(1.0, kg), fh = std::ldexp(1.0, kh);
            const uint32_t b = part.begin[c.node], cnt = part.count[c.node];
            for (uint32_t i = 0; i < cnt; ++i) {
                const uint32_t row = part.indices[b + i];
                sg += std::llrint((double)rgrad[row] * fg);
                sh += std::llrint((double)rhess[row] * fh);
            }
            g = (double)sg * std::ldexp(1.0, -kg);
            h = (double)sh * std::ldexp(1.0, -kh);
        }
        float w = leaf_weight(tc.sc.gp, g, h);
        tree.is_leaf[c.tree_node] = 1;
        tree.leaf[c.tree_node] = w;
        tree.cover[c.tree_node] = f64_to_f32(h);
        tree.grad_sum[c.tree_node] = g;
        tree.hess_sum[c.tree_node] = h;
        record_leaf(c.tree_node, c.node, w);
        pool.release(c.node);
    }

    // grower.rs:576-650 apply_split_to_builder
    std::pair<uint32_t, uint32_t> apply_split(uint32_t node, const Split& s) {
        uint32_t orig = ds->col_feature[s.feature];
        const BinMapper& m = ds->mappers[orig];
        uint32_t l = tree.alloc(), r = tree.alloc();
        tree.split_index[node] = orig;
        tree.left[node] = l;
        tree.right[node] = r;
        tree.is_leaf[node] = 0;
        if (!s.categorical) {
            float upper = f64_to_f32(m.bin_to_value(s.bin));
            tree.threshold[node] = next_up_f32(upper);
            tree.default_left[node] = s.default_left ? 1 : 0;
            tree.split_type[node] = 0;
            tree.split_bin[node] = s.bin;
            return {l, r};
        }
        tree.threshold[node] = 0.0f;
        tree.default_left[node] = s.default_left ? 0 : 1;  // inverted
        tree.split_type[node] = 1;
        tree.cat_nodes.push_back({node, categories_to_bitset(s.left_cats)});
        return {r, l};  // children swapped
    }

    void grow(const float* g, const float* h, bool record_leaves) {
        grad = g;
        hess = h;
        uint64_t n = ds->n;
        pool.reset_mappings();
        part.reset(n);
        tree = Tree();
        for (auto& v : last_leaf) v = std::numeric_limits<float>::quiet_NaN();
        leaf_map.clear();
        tree.alloc();  // root = 0
        build_histogram(0);
        auto tot = sum_gradients(0);
        cs_begin_tree();
        const uint32_t root_cnt = rmask ? n_sampled : (uint32_t)n;
        Split root = find(0, tot.first, tot.second, root_cnt, 0);
        std::vector<Candidate> cur, next, heap;
        Candidate rc{0, 0, 0, root, tot.first, tot.second, root_cnt};
        uint32_t depth = 0, n_leaves = 1;
        if (tc.leafwise)
            heap.push_back(rc);
        else
            cur.push_back(rc);
        auto heap_pop = [&]() {  // max by (gain, node) (expansion.rs:308-320)
            size_t bi = 0;
            for (size_t i = 1; i < heap.size(); ++i) {
                const Candidate& a = heap[i];
                const Candidate& b = heap[bi];
                bool greater = a.split.gain > b.split.gain || (a.split.gain == b.split.gain && a.node > b.node);
                if (greater) bi = i;
            }
            Candidate c = heap[bi];
            heap.erase(heap.begin() + bi);
            return c;
        };
        auto push = [&](const Candidate& c) {
            if (tc.leafwise)
                heap.push_back(c);
            else
                next.push_back(c);
        };
        auto process = [&](Candidate c) {  // grower.rs:346-481
            bool expand = c.split.valid() && !(c.split.gain <= tc.sc.gp.min_gain);
            if (!expand) {
                make_leaf(c);
                return;
            }
            tree.gain[c.tree_node] = c.split.gain;
            tree.cover[c.tree_node] = f64_to_f32(c.h * tc.sc.gp.sh);
            tree.grad_sum[c.tree_node] = c.g * tc.sc.gp.sg;
            tree.hess_sum[c.tree_node] = c.h * tc.sc.gp.sh;
            auto lr = apply_split(c.tree_node, c.split);
            // partition (partition.rs:296-382)
            uint32_t col = c.split.feature;
            const uint16_t* bins = ds->col_bins[col].data();
            bool hm = ds->col_missing[col] != 0;
            uint32_t db = ds->col_default[col];
            const Split& s = c.split;
            uint32_t lc, rcnt;
            uint32_t right_node = part.split(c.node, [&](uint32_t row) {
                uint32_t bin = bins[row];
                if (hm && bin == db) return s.default_left;
                if (!s.categorical) return bin <= s.bin;
                return std::binary_search(s.left_cats.begin(), s.left_cats.end(), bin);
            }, lc, rcnt);
            if (rmask) {  // counts of the sampled rows
                lc = sampled_in(c.node);
                rcnt = sampled_in(right_node);
            }
            uint32_t left_node = c.node, parent = c.node;
            bool left_small = lc <= rcnt;
            uint32_t small = left_small ? left_node : right_node;
            uint32_t large = left_small ? right_node : left_node;
            uint32_t small_cnt = left_small ? lc : rcnt, large_cnt = left_small ? rcnt : lc;
            if (pool.resolve(parent) >= 0) {
                pool.pin(parent);
                pool.move_mapping(parent, large);
                build_histogram(small);
                pool.subtract(large, small);
                pool.unpin(large);
            } else {
                build_histogram(left_node);
                build_histogram(right_node);
            }
            auto ss = sum_gradients(small);
            double lg = c.g - ss.first, lh = c.h - ss.second;
            Split s_small = find(small, ss.first, ss.second, small_cnt, c.depth + 1);
            Split s_large = find(large, lg, lh, large_cnt, c.depth + 1);
            Candidate cl, cr;
            if (left_node == small)
                cl = {left_node, lr.first, c.depth + 1, s_small, ss.first, ss.second, small_cnt};
            else
                cl = {left_node, lr.first, c.depth + 1, s_large, lg, lh, large_cnt};
            if (right_node == small)
                cr = {right_node, lr.second, c.depth + 1, s_small, ss.first, ss.second, small_cnt};
            else
                cr = {right_node, lr.second, c.depth + 1, s_large, lg, lh, large_cnt};
            push(cl);
            push(cr);
        };
        if (tc.leafwise) {
            while (n_leaves < tc.max_leaves && !heap.empty()) {
                Candidate c = heap_pop();
                n_leaves += 1;
                process(c);
            }
            while (!heap.empty()) make_leaf(heap_pop());
        } else {
            while (depth < tc.max_depth && !cur.empty()) {
                std::vector<Candidate> level;
                level.swap(cur);
                for (auto& c : level) process(c);
                cur.swap(next);
                next.clear();
                depth += 1;
            }
            for (auto& c : cur) make_leaf(c);
        }
        // apply_learning_rate (mutable_tree.rs:258-265)
        for (size_t i = 0; i < tree.leaf.size(); ++i)
            if (tree.is_leaf[i]) tree.leaf[i] = tree.leaf[i] * tc.learning_rate;
        tree.freeze();
        if (record_leaves) {
            tree.row_leaf.assign(n, 0);
            for (auto& lm : leaf_map) {
                uint32_t b = part.begin[lm.second], c = part.count[lm.second];
                for (uint32_t i = 0; i < c; ++i) tree.row_leaf[part.indices[b + i]] = lm.first;
            }
        }
    }

    // Leaf renewing (trainer.rs:283-313, objectives/mod.rs:352-409): each
    // leaf's value becomes the alpha-quantile of the residuals y - pred of
    // its (sampled) rows, in partition order, times the learning rate.
    void renew_leaves(const float* y, const float* w, const float* pred, float alpha) {
        std::vector<float> v, wt;
        for (const auto& lm : leaf_map) {
            const uint32_t b = part.begin[lm.second], c = part.count[lm.second];
            v.clear();
            wt.clear();
            for (uint32_t i = 0; i < c; ++i) {
                const uint32_t row = part.indices[b + i];
                if (rmask && !rmask[row]) continue;
                v.push_back(y[row] - pred[row]);
                if (w) wt.push_back(w[row]);
            }
            if (v.empty()) continue;
            const float q = w ? weighted_quantile(v, wt, alpha) : unweighted_quantile(v, alpha);
            if (std::isnan(q)) continue;
            const float sv = q * tc.learning_rate;
            tree.leaf[lm.first] = sv;
            last_leaf[lm.second] = sv;
        }
    }

    // grower.rs:208-219 update_predictions_from_last_tree
    void update_predictions(float* pred) {
        for (size_t node = 0; node < last_leaf.size(); ++node) {
            float v = last_leaf[node];
            if (std::isnan(v)) continue;
            uint32_t b = part.begin[node], c = part.count[node];
            for (uint32_t i = 0; i < c; ++i) pred[part.indices[b + i]] += v;
        }
    }
};

// ---------------------------------------------------------------------------
// Quantised gradients (not in the reference: the int8 / int16 training mode of
// the GPU engine). Philox4x32-10 counter-based generator as published by
// Salmon, Moraes, Dror and Shaw, "Parallel Random Numbers: As Easy as 1, 2, 3"
// (SC 2011); stochastic rounding q = floor(v * Q / max|v| + u), u in [0, 1).
// ---------------------------------------------------------------------------

void philox4x32_10(const uint32_t in[4], const uint32_t key[2], uint32_t out[4]) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    uint32_t c0 = in[0], c1 = in[1], c2 = in[2], c3 = in[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)M0 * c0, p1 = (uint64_t)M1 * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += W0;
        k1 += W1;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

const uint32_t QUANT_STREAM = 0x51A7E5EDu;  // fourth counter word of the rounding stream

inline int32_t quant_max(int precision) { return precision == BST_PRECISION_Q8 ? 127 : 32767; }

inline float max_abs_finite(const float* v, uint64_t n) {
    float m = 0.0f;
    for (uint64_t i = 0; i < n; ++i) {
        const float a = std::fabs(v[i]);
        if (a <= 3.4e38f && a > m) m = a;  // the engine's scale ignores |v| > 3.4e38
    }
    return m;
}

int fixed_point_k(float m, uint64_t n) {
    if (!(m > 0.0f)) return 0;
    int e, en;
    std::frexp((double)m, &e);
    std::frexp((double)n, &en);
    int B = 38;
    if (61 - en < B) B = 61 - en;
    int k = B - e;
    return k > 1000 ? 1000 : (k < -1000 ? -1000 : k);
}

// steps = (Q / max|g|, Q / max|h|, max|g| / Q, max|h| / Q); all zero for a
// zero (or non-finite) maximum
void quantize(const float* g, const float* h, uint64_t n, int precision, uint64_t seed, uint32_t round,
              uint32_t output, int32_t* qg, int32_t* qh, double* steps) {
    const int32_t Q = quant_max(precision);
    const float mg = max_abs_finite(g, n), mh = max_abs_finite(h, n);
    const double ig = mg > 0.0f ? (double)Q / (double)mg : 0.0;
    const double ih = mh > 0.0f ? (double)Q / (double)mh : 0.0;
    steps[0] = ig;
    steps[1] = ih;
    steps[2] = mg > 0.0f ? (double)mg / (double)Q : 0.0;
    steps[3] = mh > 0.0f ? (double)mh / (double)Q : 0.0;
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    for (uint64_t i = 0; i < n; ++i) {
        const uint32_t ctr[4] = {(uint32_t)i, output, round, QUANT_STREAM};
        uint32_t r[4];
        philox4x32_10(ctr, key, r);
        const double ug = (double)r[0] * 0x1p-32, uh = (double)r[1] * 0x1p-32;
        double xg = (double)g[i] * ig;
        xg = xg + ug;
        double xh = (double)h[i] * ih;
        xh = xh + uh;
        double fg = std::floor(xg), fh = std::floor(xh);
        if (!(fg >= -Q)) fg = -Q;  // also maps NaN to -Q
        if (fg > Q) fg = Q;
        if (!(fh >= -Q)) fh = -Q;
        if (fh > Q) fh = Q;
        qg[i] = (int32_t)fg;
        qh[i] = (int32_t)fh;
    }
}

}  // namespace

struct orc_model {
    uint32_t n_groups = 1;
    uint32_t n_features = 0;
    int objective = 0;
    std::vector<float> base;
    std::vector<Tree> trees;
    std::vector<float> train_pred;
    double train_seconds = 0, binning_seconds = 0;
    std::vector<double> tree_seconds;  // per tree: growth + prediction update (+ gradients of its round)
};

// ---------------------------------------------------------------------------
// Prediction (inference/gbdt/predictor.rs:197-302, model/transform.rs:61-115)
// ---------------------------------------------------------------------------

namespace {

inline float sigmoid_t(float x) {  // transform.rs:106-115
    float c = x < -500.0f ? -500.0f : (x > 500.0f ? 500.0f : x);
    if (c >= 0.0f) return 1.0f / (1.0f + exp_f32(-c));
    float e = exp_f32(c);
    return e / (1.0f + e);
}

void transform(int t, float* p, uint32_t G, uint64_t n) {
    if (t == 1) {
        for (uint64_t i = 0; i < (uint64_t)G * n; ++i) p[i] = sigmoid_t(p[i]);
    } else if (t == 2) {
        for (uint64_t i = 0; i < n; ++i) {  // softmax_inplace (transform.rs:83-101)
            float mx = -std::numeric_limits<float>::infinity();
            for (uint32_t g = 0; g < G; ++g) mx = std::fmax(mx, p[g * n + i]);
            float sum = 0.0f;
            for (uint32_t g = 0; g < G; ++g) {
                float e = exp_f32(p[g * n + i] - mx);
                p[g * n + i] = e;
                sum += e;
            }
            if (sum > 0.0f)
                for (uint32_t g = 0; g < G; ++g) p[g * n + i] /= sum;
        }
    }
}

int transform_of(int objective) { return objective == BST_OBJ_LOGISTIC ? 1 : (objective == BST_OBJ_SOFTMAX ? 2 : 0); }

void predict_impl(const orc_model* m, const float* x, uint64_t n, bool sample_major, uint64_t F,
                  bool raw, int omp_threads, float* out) {
    uint32_t G = m->n_groups;
    for (uint32_t g = 0; g < G; ++g)
        for (uint64_t i = 0; i < n; ++i) out[g * n + i] = m->base[g];
    auto row = [&](int64_t i) {
        const float* xr = sample_major ? x + (uint64_t)i * F : x + i;
        uint64_t stride = sample_major ? 1 : n;
        for (const Tree& t : m->trees) {
            uint32_t leaf = t.traverse(xr, stride);
            out[(uint64_t)t.group * n + i] += t.leaf[leaf];
        }
    };
#ifdef _OPENMP
    if (omp_threads > 1) {
#pragma omp parallel for num_threads(omp_threads) schedule(static, 64)
        for (int64_t i = 0; i < (int64_t)n; ++i) row(i);
    } else
#endif
        for (int64_t i = 0; i < (int64_t)n; ++i) row(i);
    if (!raw) transform(transform_of(m->objective), out, G, n);
}

double metric_impl(int metric, const ObjP& op, const float* p, uint32_t G, uint64_t n, const float* y,
                   const float* w) {
    if (n == 0) return 0.0;
    const double EPS = 1e-15;
    if (metric == BST_METRIC_MAE) {  // metrics/regression.rs:55-87
        double sum = 0.0;
        for (uint32_t g = 0; g < G; ++g) {
            double sa = 0, sw = 0;
            for (uint64_t i = 0; i < n; ++i) {
                const double wi = (double)w_at(w, i);
                sa = sa + wi * std::fabs((double)p[g * n + i] - (double)y[i]);
                sw = sw + wi;
            }
            sum += sw > 0.0 ? sa / sw : 0.0;
        }
        return sum / (double)G;
    }
    if (metric == BST_METRIC_MAPE) {  // metrics/regression.rs:89-124
        double sa = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const double pp = (double)p[i], l = (double)y[i], wi = (double)w_at(w, i);
            sa = sa + wi * (std::fabs(pp - l) / std::fmax(std::fabs(l), EPS));
            sw = sw + wi;
        }
        return sw > 0.0 ? (sa / sw) * 100.0 : 0.0;
    }
    if (metric == BST_METRIC_QUANTILE) {  // metrics/regression.rs:126-174
        double tl = 0, tw = 0;
        for (uint32_t q = 0; q < G; ++q) {
            const double a = (double)op.alpha_at(q);
            double l = 0, sw = 0;
            for (uint64_t i = 0; i < n; ++i) {
                const double r = (double)y[i] - (double)p[q * n + i], wi = (double)w_at(w, i);
                const double loss = r >= 0.0 ? a * r : (1.0 - a) * (-r);
                l = l + wi * loss;
                sw = sw + wi;
            }
            tl = tl + l;
            tw = tw + sw;
        }
        return tw > 0.0 ? tl / tw : 0.0;
    }
    if (metric == BST_METRIC_HUBER) {  // metrics/regression.rs:216-245
        const double delta = (double)op.delta;
        double sl = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const double r = std::fabs((double)p[i] - (double)y[i]), wi = (double)w_at(w, i);
            const double loss = r <= delta ? 0.5 * r * r : delta * (r - 0.5 * delta);
            sl = sl + wi * loss;
            sw = sw + wi;
        }
        return sw > 0.0 ? sl / sw : 0.0;
    }
    if (metric == BST_METRIC_POISSON) {  // metrics/regression.rs:176-210
        const double E = 1e-9;
        double sd = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const double yy = (double)y[i], mu = std::fmax((double)p[i], E), wi = (double)w_at(w, i);
            const double dev = yy > E ? 2.0 * (yy * std::log(yy / mu) - (yy - mu)) : 2.0 * mu;
            sd = sd + wi * dev;
            sw = sw + wi;
        }
        return sw > 0.0 ? sd / sw : 0.0;
    }
    if (metric == BST_METRIC_MARGIN_ACCURACY) {  // metrics/classification.rs:85-118, threshold 0
        double sc = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const float pc = p[i] >= 0.0f ? 1.0f : 0.0f;
            const double c = std::fabs(pc - y[i]) < 0.5f ? 1.0 : 0.0, wi = (double)w_at(w, i);
            sc = sc + wi * c;
            sw = sw + wi;
        }
        return sw > 0.0 ? sc / sw : 0.0;
    }
    if (metric == BST_METRIC_RMSE) {  // metrics/regression.rs:17-45
        double sum = 0.0;
        for (uint32_t g = 0; g < G; ++g) {
            double ss = 0, sw = 0;
            for (uint64_t i = 0; i < n; ++i) {
                double d = (double)p[g * n + i] - (double)y[i];
                double wi = (double)w_at(w, i);
                ss = ss + wi * d * d;
                sw = sw + wi;
            }
            sum += sw > 0.0 ? std::sqrt(ss / sw) : 0.0;
        }
        return sum / (double)G;
    }
    if (metric == BST_METRIC_LOGLOSS) {  // metrics/classification.rs:13-40
        double sl = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            double pp = clamp64((double)p[i], EPS, 1.0 - EPS);
            double l = (double)y[i];
            double loss = -(l * std::log(pp) + (1.0 - l) * std::log(1.0 - pp));
            double wi = (double)w_at(w, i);
            sl = sl + wi * loss;
            sw = sw + wi;
        }
        return sw > 0.0 ? sl / sw : 0.0;
    }
    if (metric == BST_METRIC_MLOGLOSS) {  // metrics/classification.rs:332-360
        double sl = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t c = sat_usize(std::round(y[i]));
            double pp = c < G ? (double)p[c * n + i] : EPS;
            pp = clamp64(pp, EPS, 1.0 - EPS);
            double wi = (double)w_at(w, i);
            sl = sl + wi * -std::log(pp);
            sw = sw + wi;
        }
        return sw > 0.0 ? sl / sw : 0.0;
    }
    return 0.0;
}

int validate_cfg(const bst_config& c) {  // model/gbdt/config.rs:252-310
    if (c.learning_rate <= 0.0f) {
        g_err = "learning_rate must be positive, got " + std::to_string(c.learning_rate);
        return BST_ERR_CONFIG;
    }
    if (c.n_trees == 0) {
        g_err = "n_trees must be at least 1";
        return BST_ERR_CONFIG;
    }
    const float* ratios[3] = {&c.subsample, &c.colsample_bytree, &c.colsample_bylevel};
    const char* rn[3] = {"subsample", "colsample_bytree", "colsample_bylevel"};
    for (int i = 0; i < 3; ++i)
        if (*ratios[i] <= 0.0f || *ratios[i] > 1.0f) {
            g_err = std::string(rn[i]) + " must be in (0, 1], got " + std::to_string(*ratios[i]);
            return BST_ERR_CONFIG;
        }
    const float* regs[4] = {&c.lambda, &c.alpha, &c.min_child_weight, &c.min_gain};
    const char* gn[4] = {"lambda", "alpha", "min_child_weight", "min_gain"};
    for (int i = 0; i < 4; ++i)
        if (*regs[i] < 0.0f) {
            g_err = std::string(gn[i]) + " must be non-negative, got " + std::to_string(*regs[i]);
            return BST_ERR_CONFIG;
        }
    if (c.objective == BST_OBJ_PINBALL) {
        if (c.n_quantiles == 0 || !c.quantile_alpha) {
            g_err = "pinball loss needs at least one quantile";
            return BST_ERR_CONFIG;
        }
        for (uint32_t i = 0; i < c.n_quantiles; ++i)
            if (!(c.quantile_alpha[i] > 0.0f && c.quantile_alpha[i] < 1.0f)) {
                g_err = "quantile alpha must be in (0, 1)";
                return BST_ERR_CONFIG;
            }
    }
    if (c.objective == BST_OBJ_PSEUDO_HUBER && !(c.huber_delta > 0.0f)) {
        g_err = "huber_delta must be positive";
        return BST_ERR_CONFIG;
    }
    if (c.goss_top_rate != 0.0f || c.goss_other_rate != 0.0f) {
        if (!(c.goss_top_rate > 0.0f) || !(c.goss_other_rate > 0.0f)) {
            g_err = "GOSS top_rate and other_rate must be positive";
            return BST_ERR_CONFIG;
        }
        if (c.goss_top_rate + c.goss_other_rate > 1.0f) {
            g_err = "top_rate + other_rate must be <= 1.0";
            return BST_ERR_CONFIG;
        }
        if (std::fabs(c.subsample - 1.0f) >= 1e-6f) {
            g_err = "GOSS and subsample < 1 cannot be combined";
            return BST_ERR_CONFIG;
        }
    }
    return 0;
}

SplitterCfg splitter_cfg(const bst_config& c, uint32_t n_threads, int omp) {
    SplitterCfg sc;
    sc.gp.lambda = c.lambda;
    sc.gp.alpha = c.alpha;
    sc.gp.min_gain = c.min_gain;
    sc.gp.min_child_weight = c.min_child_weight;
    sc.gp.min_samples_leaf = c.min_samples_leaf;
    sc.max_onehot_cats = c.max_onehot_cats;
    sc.parallel = n_threads != 1;  // Parallelism::from_threads (utils.rs:152-158)
    sc.omp_threads = omp < 1 ? 1 : omp;
    return sc;
}

}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

// GBDTConfig's builder defaults (model/gbdt/config.rs:111-226) and the
// binning defaults (data/binned/feature_analysis.rs:29-63); GPU-only fields
// are zero.
void orc_config_default(bst_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->objective = BST_OBJ_SQUARED;
    c->metric = BST_METRIC_DEFAULT;
    c->n_trees = 100;
    c->learning_rate = 0.3f;
    c->growth_strategy = BST_GROWTH_DEPTHWISE;
    c->max_depth = 6;
    c->max_leaves = 31;
    c->max_onehot_cats = 4;
    c->lambda = 1.0f;
    c->min_child_weight = 1.0f;
    c->min_samples_leaf = 1;
    c->subsample = 1.0f;
    c->colsample_bytree = 1.0f;
    c->colsample_bylevel = 1.0f;
    c->max_bins = 256;
    c->sparsity_threshold = 0.9f;
    c->enable_bundling = 1;
    c->binning_sample_cnt = 200000;
    c->early_stopping_rounds = -1;
    c->cache_size = 8;
    c->seed = 42;
    c->huber_delta = 1.0f;
}

int orc_synth_regression(uint64_t n, uint64_t F, uint64_t n_inf, uint64_t seed, uint64_t stream, float* x,
                         float* y) {
    return synthgen::regression(n, F, n_inf, seed, stream, x, y);
}
int orc_synth_binary(uint64_t n, uint64_t F, uint64_t n_nan_cols, uint64_t seed, uint64_t stream, float* x,
                     float* y) {
    return synthgen::binary(n, F, n_nan_cols, seed, stream, x, y);
}
int orc_synth_multiclass(uint64_t n, uint64_t n_num, uint64_t n_cat, uint64_t C, uint64_t seed, uint64_t stream,
                         float* x, float* y) {
    return synthgen::multiclass(n, n_num, n_cat, C, seed, stream, x, y);
}

int orc_bin(const float* x, uint64_t F, uint64_t n, const uint32_t* cat_idx, uint32_t n_cat,
            const bst_config* cfg, orc_binned** out) {
    orc_binned* b = new orc_binned();
    int rc = build_binned(x, F, n, cat_idx, n_cat, *cfg, *b);
    if (rc) {
        delete b;
        return rc;
    }
    *out = b;
    return 0;
}
void orc_binned_free(orc_binned* b) { delete b; }
uint32_t orc_binned_n_columns(const orc_binned* b) { return (uint32_t)b->col_feature.size(); }
void orc_binned_column_info(const orc_binned* b, uint32_t col, uint32_t* feature, uint32_t* n_bins,
                            int32_t* is_cat, int32_t* has_missing, uint32_t* default_bin) {
    if (feature) *feature = b->col_feature[col];
    if (n_bins) *n_bins = b->col_nbins[col];
    if (is_cat) *is_cat = b->col_cat[col];
    if (has_missing) *has_missing = b->col_missing[col];
    if (default_bin) *default_bin = b->col_default[col];
}
void orc_binned_column_bounds(const orc_binned* b, uint32_t col, double* out) {
    const BinMapper& m = b->mappers[b->col_feature[col]];
    for (uint32_t i = 0; i < m.n_bins; ++i) out[i] = m.categorical ? (double)m.cats[i] : m.bounds[i];
}
void orc_binned_column_bins(const orc_binned* b, uint32_t col, uint16_t* out) {
    std::memcpy(out, b->col_bins[col].data(), b->n * sizeof(uint16_t));
}

uint32_t orc_value_to_bin(const double* bounds, uint32_t n_bounds, int32_t missing_type,
                          uint32_t default_bin, int32_t is_cat, const int32_t* cats, uint32_t n_cats,
                          double value) {
    BinMapper m = is_cat ? BinMapper::categorical_from(std::vector<int32_t>(cats, cats + n_cats), missing_type, default_bin)
                         : BinMapper::numerical(std::vector<double>(bounds, bounds + n_bounds), missing_type, default_bin);
    return m.value_to_bin(value);
}

double orc_gain_full(double gl, double hl, double gr, double hr, double gp, double hp, float lambda,
                     float min_gain) {
    double l = (double)lambda;
    double sl = gl * gl / (hl + l), sr = gr * gr / (hr + l), sp = gp * gp / (hp + l);
    return (double)f64_to_f32(0.5 * (sl + sr - sp) - (double)min_gain);
}
float orc_leaf_weight(double g, double h, float lambda, float alpha) {
    GainParams p;
    p.lambda = lambda;
    p.alpha = alpha;
    return leaf_weight(p, g, h);
}
int orc_is_valid_split(double hl, double hr, uint32_t cl, uint32_t cr, float mcw, uint32_t msl) {
    GainParams p;
    p.min_child_weight = mcw;
    p.min_samples_leaf = msl;
    return is_valid_split(p, hl, hr, cl, cr) ? 1 : 0;
}

void orc_histogram_build(const uint16_t* bins, const uint32_t* n_bins, uint32_t F, uint64_t n,
                         const float* grad, const float* hess, const uint32_t* rows, uint64_t n_rows,
                         double* out) {
    uint64_t off = 0;
    uint64_t cnt = rows ? n_rows : n;
    for (uint32_t f = 0; f < F; ++f) {
        double* h = out + 2 * off;
        for (uint32_t b = 0; b < n_bins[f]; ++b) h[2 * b] = h[2 * b + 1] = 0.0;
        for (uint64_t i = 0; i < cnt; ++i) {
            uint64_t r = rows ? rows[i] : i;
            uint16_t b = bins[(uint64_t)f * n + r];
            h[2 * b] += (double)grad[r];
            h[2 * b + 1] += (double)hess[r];
        }
        off += n_bins[f];
    }
}

void orc_find_split(const double* hist, const uint32_t* n_bins, const int32_t* is_cat,
                    const int32_t* has_missing, uint32_t F, double pg, double ph, uint32_t pc,
                    const bst_config* cfg, uint32_t n_threads, bst_split* out) {
    std::vector<uint32_t> offs(F), nb(n_bins, n_bins + F);
    std::vector<uint8_t> ic(F), hm(F);
    uint32_t o = 0, tot = 0;
    for (uint32_t f = 0; f < F; ++f) {
        offs[f] = o;
        o += n_bins[f];
        ic[f] = is_cat[f] ? 1 : 0;
        hm[f] = has_missing[f] ? 1 : 0;
    }
    tot = o;
    std::vector<HBin> h(tot);
    for (uint32_t i = 0; i < tot; ++i) h[i] = {hist[2 * i], hist[2 * i + 1]};
    Split s = find_split(h.data(), offs.data(), nb.data(), ic.data(), hm.data(), F, pg, ph, pc,
                         splitter_cfg(*cfg, n_threads, 1));
    std::memset(out, 0, sizeof(*out));
    out->feature = s.feature;
    out->gain = s.gain;
    out->default_left = s.default_left;
    out->is_categorical = s.categorical;
    out->bin = s.bin;
    for (uint32_t c : s.left_cats)
        if (c < 256) out->left_cats[c >> 6] |= 1ULL << (c & 63);
}

void orc_gradients(int32_t obj, uint32_t G, const float* preds, const float* y, const float* w,
                   uint64_t n, float* grad, float* hess) {
    gradients(obj, ObjP(), G, preds, y, w, n, grad, hess);
}
void orc_base_score(int32_t obj, uint32_t G, const float* y, const float* w, uint64_t n, float* out) {
    base_score(obj, ObjP(), G, y, w, n, out);
}
void orc_gradients_cfg(const bst_config* c, uint32_t G, const float* preds, const float* y, const float* w,
                       uint64_t n, float* grad, float* hess) {
    gradients(c->objective, ObjP::of(*c), G, preds, y, w, n, grad, hess);
}
void orc_base_score_cfg(const bst_config* c, uint32_t G, const float* y, const float* w, uint64_t n, float* out) {
    base_score(c->objective, ObjP::of(*c), G, y, w, n, out);
}
double orc_metric_cfg(int32_t metric, const bst_config* c, const float* p, uint32_t G, uint64_t n, const float* y,
                      const float* w) {
    return metric_impl(metric, ObjP::of(*c), p, G, n, y, w);
}
uint64_t orc_goss(float* g, float* h, uint64_t n, float top_rate, float other_rate, uint64_t seed, uint32_t calls,
                  uint8_t* mask) {
    OracleRowSampler rs(seed);
    std::vector<uint8_t> m;
    uint64_t k = 0;
    for (uint32_t c = 0; c < calls; ++c) k = rs.goss(g, h, n, top_rate, other_rate, m);
    std::copy(m.begin(), m.end(), mask);
    return k;
}
float orc_leaf_quantile(const float* v, const float* w, uint64_t n, float alpha) {
    std::vector<float> vv(v, v + n), ww;
    if (w) ww.assign(w, w + n);
    return w ? weighted_quantile(vv, ww, alpha) : unweighted_quantile(vv, alpha);
}
void orc_transform(int32_t t, float* p, uint32_t G, uint64_t n) { transform(t, p, G, n); }
double orc_metric(int32_t metric, const float* p, uint32_t G, uint64_t n, const float* y, const float* w) {
    return metric_impl(metric, ObjP(), p, G, n, y, w);
}
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    philox4x32_10(ctr, key, out);
}
void orc_quantize(const float* g, const float* h, uint64_t n, int32_t precision, uint64_t seed, uint32_t round,
                  uint32_t output, int32_t* qg, int32_t* qh, double* steps) {
    quantize(g, h, n, precision, seed, round, output, qg, qh, steps);
}

int orc_train_limited(const float* x, uint64_t F, uint64_t n, const float* y, uint32_t y_rows,
                      const float* w, const uint32_t* cat_idx, uint32_t n_cat, const bst_config* cfgp,
                      uint32_t n_threads, int record_leaves, int omp_threads, uint32_t max_trees,
                      orc_model** out) {
    const bst_config& cfg = *cfgp;
    int rc = validate_cfg(cfg);
    if (rc) return rc;
    if (!y || y_rows == 0) {
        g_err = "dataset must have targets for training";
        return BST_ERR_MISSING_TARGETS;
    }
    if (cfg.early_stopping_rounds >= 0) {
        g_err = "early stopping is outside this restatement";
        return BST_ERR_UNSUPPORTED;
    }
    if (cfg.objective == BST_OBJ_SOFTMAX && cfg.n_classes < 2) {
        g_err = "softmax needs n_classes >= 2";
        return BST_ERR_CONFIG;
    }
    const bool goss_on = cfg.goss_top_rate > 0.0f;
    if (goss_on && n < 2) {
        g_err = "GOSS needs at least 2 rows";
        return BST_ERR_CONFIG;
    }
    const ObjP op = ObjP::of(cfg);
    auto t0 = std::chrono::steady_clock::now();
    orc_binned b;
    rc = build_binned(x, F, n, cat_idx, n_cat, cfg, b, omp_threads);
    if (rc) return rc;
    auto t1 = std::chrono::steady_clock::now();
    orc_model* m = new orc_model();
    m->objective = cfg.objective;
    m->n_groups = cfg.objective == BST_OBJ_SOFTMAX ? cfg.n_classes
                                                   : (cfg.objective == BST_OBJ_PINBALL ? cfg.n_quantiles : 1);
    m->n_features = (uint32_t)F;
    m->binning_seconds = std::chrono::duration<double>(t1 - t0).count();
    uint32_t G = m->n_groups;
    // trainer.rs:162-401
    m->base.resize(G);
    base_score(cfg.objective, op, G, y, w, n, m->base.data());
    m->train_pred.resize((size_t)G * n);
    for (uint32_t g = 0; g < G; ++g) std::fill(m->train_pred.begin() + g * n, m->train_pred.begin() + (g + 1) * n, m->base[g]);
    std::vector<float> grad((size_t)G * n), hess((size_t)G * n);
    TrainCfg tc;
    tc.sc = splitter_cfg(cfg, n_threads, omp_threads);
    tc.learning_rate = cfg.learning_rate;
    tc.leafwise = cfg.growth_strategy == BST_GROWTH_LEAFWISE;
    tc.max_depth = cfg.max_depth;
    tc.max_leaves = cfg.max_leaves;
    tc.cache_size = cfg.cache_size;
    tc.colsample_bytree = cfg.colsample_bytree;
    tc.colsample_bylevel = cfg.colsample_bylevel;
    tc.seed = cfg.seed;
    Grower gr;
    gr.init(&b, tc);
    uint32_t n_rounds = cfg.n_trees;
    uint32_t built = 0;
    const bool quant = cfg.precision != BST_PRECISION_FP32;
    std::vector<int32_t> qg, qh;
    std::vector<float> fqg, fqh;
    // row sampling (config.rs:329-330: a rate within 1e-6 of 1 samples nothing)
    // GOSS (row.rs:214-280) from round floor(1 / learning_rate) on
    std::unique_ptr<OracleRowSampler> row_sampler;
    std::vector<uint8_t> row_mask;
    const bool uniform_on = std::fabs(cfg.subsample - 1.0f) >= 1e-6f;
    if (uniform_on || goss_on) row_sampler = std::make_unique<OracleRowSampler>(cfg.seed);
    const uint64_t goss_warmup = (uint64_t)(1.0f / cfg.learning_rate);
    const bool renew = cfg.objective == BST_OBJ_ABSOLUTE || cfg.objective == BST_OBJ_PINBALL;
    if (quant) {
        qg.resize(n);
        qh.resize(n);
        fqg.resize(n);
        fqh.resize(n);
    }
    for (uint32_t round = 0; round < n_rounds && built < max_trees; ++round) {
        auto tr0 = std::chrono::steady_clock::now();
        gradients(cfg.objective, op, G, m->train_pred.data(), y, w, n, grad.data(), hess.data());
        for (uint32_t o = 0; o < G && built < max_trees; ++o) {
            gr.rmask = nullptr;
            gr.n_sampled = (uint32_t)n;
            const bool sampled = uniform_on || (goss_on && round >= goss_warmup);
            if (sampled) {  // row.rs:141-280: rows outside the sample leave the tree (zero grad/hess)
                if (goss_on)
                    gr.n_sampled = (uint32_t)row_sampler->goss(grad.data() + (size_t)o * n, hess.data() + (size_t)o * n,
                                                               n, cfg.goss_top_rate, cfg.goss_other_rate, row_mask);
                else
                    gr.n_sampled = (uint32_t)row_sampler->sample(n, cfg.subsample, row_mask);
                gr.rmask = row_mask.data();
                for (uint64_t i = 0; i < n; ++i)
                    if (!row_mask[i]) grad[(size_t)o * n + i] = hess[(size_t)o * n + i] = 0.0f;
            }
            const float* go = grad.data() + (size_t)o * n;
            const float* ho = hess.data() + (size_t)o * n;
            if (quant) {
                double steps[4];
                quantize(go, ho, n, cfg.precision, cfg.seed, round, o, qg.data(), qh.data(), steps);
                for (uint64_t i = 0; i < n; ++i) {
                    fqg[i] = (float)qg[i];
                    fqh[i] = (float)qh[i];
                }
                gr.tc.sc.gp.sg = steps[2];
                gr.tc.sc.gp.sh = steps[3];
                gr.kg = fixed_point_k(max_abs_finite(go, n), n);
                gr.kh = fixed_point_k(max_abs_finite(ho, n), n);
                gr.rgrad = go;
                gr.rhess = ho;
                gr.cs_round = round;
                gr.cs_output = o;
                gr.grow(fqg.data(), fqh.data(), record_leaves != 0);
            } else {
                gr.cs_round = round;
                gr.cs_output = o;
                gr.grow(go, ho, record_leaves != 0);
            }
            if (renew) gr.renew_leaves(y, w, m->train_pred.data() + (size_t)o * n, op.alpha_at(o));
            gr.update_predictions(m->train_pred.data() + (size_t)o * n);
            gr.tree.group = o;
            m->trees.push_back(std::move(gr.tree));
            gr.tree = Tree();
            ++built;
            auto tr1 = std::chrono::steady_clock::now();
            m->tree_seconds.push_back(std::chrono::duration<double>(tr1 - tr0).count());
            tr0 = tr1;
        }
    }
    m->train_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
    *out = m;
    return 0;
}

int orc_train(const float* x, uint64_t F, uint64_t n, const float* y, uint32_t y_rows, const float* w,
              const uint32_t* cat_idx, uint32_t n_cat, const bst_config* cfg, uint32_t n_threads,
              int record_leaves, int omp_threads, orc_model** out) {
    return orc_train_limited(x, F, n, y, y_rows, w, cat_idx, n_cat, cfg, n_threads, record_leaves,
                             omp_threads, UINT32_MAX, out);
}

int orc_grow_tree(const float* x, uint64_t F, uint64_t n, const float* grad, const float* hess,
                  const bst_config* cfgp, uint32_t n_threads, orc_model** out) {
    const bst_config& cfg = *cfgp;
    int rc = validate_cfg(cfg);
    if (rc) return rc;
    orc_binned b;
    rc = build_binned(x, F, n, nullptr, 0, cfg, b);
    if (rc) return rc;
    TrainCfg tc;
    tc.sc = splitter_cfg(cfg, n_threads, 1);
    tc.learning_rate = cfg.learning_rate;
    tc.leafwise = cfg.growth_strategy == BST_GROWTH_LEAFWISE;
    tc.max_depth = cfg.max_depth;
    tc.max_leaves = cfg.max_leaves;
    tc.cache_size = cfg.cache_size;
    tc.colsample_bytree = cfg.colsample_bytree;
    tc.colsample_bylevel = cfg.colsample_bylevel;
    tc.seed = cfg.seed;
    Grower gr;
    gr.init(&b, tc);
    gr.grow(grad, hess, true);
    orc_model* m = new orc_model();
    m->n_groups = 1;
    m->n_features = (uint32_t)F;
    m->base = {0.0f};
    m->train_pred.assign(n, 0.0f);
    gr.update_predictions(m->train_pred.data());
    m->trees.push_back(std::move(gr.tree));
    *out = m;
    return 0;
}

int orc_model_create(uint32_t G, uint32_t F, int32_t objective, const float* base, orc_model** out) {
    orc_model* m = new orc_model();
    m->n_groups = G;
    m->n_features = F;
    m->objective = objective;
    m->base.assign(base, base + G);
    *out = m;
    return 0;
}

int orc_model_add_tree(orc_model* m, uint32_t group, uint32_t nn, const uint32_t* si, const float* thr,
                       const uint32_t* l, const uint32_t* r, const uint8_t* dl, const uint8_t* il, const float* lv,
                       const uint8_t* st, const uint32_t* ss, const uint32_t* sz, const uint32_t* words,
                       uint32_t n_words) {
    Tree t;
    for (uint32_t i = 0; i < nn; ++i) t.alloc();
    for (uint32_t i = 0; i < nn; ++i) {
        t.split_index[i] = si[i];
        t.threshold[i] = thr[i];
        t.left[i] = l[i];
        t.right[i] = r[i];
        t.default_left[i] = dl[i];
        t.is_leaf[i] = il[i];
        t.leaf[i] = lv[i];
        t.split_type[i] = st ? st[i] : 0;
    }
    t.seg_start.assign(nn, 0);
    t.seg_size.assign(nn, 0);
    if (ss && sz) {
        t.seg_start.assign(ss, ss + nn);
        t.seg_size.assign(sz, sz + nn);
    }
    if (words) t.cat_words.assign(words, words + n_words);
    t.group = group;
    m->trees.push_back(std::move(t));
    return 0;
}

void orc_model_free(orc_model* m) { delete m; }
uint32_t orc_model_n_trees(const orc_model* m) { return (uint32_t)m->trees.size(); }
uint32_t orc_model_n_groups(const orc_model* m) { return m->n_groups; }
void orc_model_base_scores(const orc_model* m, float* out) { std::copy(m->base.begin(), m->base.end(), out); }
void orc_model_train_predictions(const orc_model* m, float* out) {
    std::copy(m->train_pred.begin(), m->train_pred.end(), out);
}
void orc_tree_info(const orc_model* m, uint32_t t, uint32_t* n_nodes, uint32_t* group, uint32_t* n_cat_words) {
    const Tree& tr = m->trees[t];
    if (n_nodes) *n_nodes = (uint32_t)tr.split_index.size();
    if (group) *group = tr.group;
    if (n_cat_words) *n_cat_words = (uint32_t)tr.cat_words.size();
}
void orc_tree_nodes(const orc_model* m, uint32_t t, uint32_t* si, float* thr, uint32_t* l, uint32_t* r,
                    uint8_t* dl, uint8_t* il, float* lv, uint8_t* st, float* gain, float* cover) {
    const Tree& tr = m->trees[t];
    size_t nn = tr.split_index.size();
    if (si) std::copy(tr.split_index.begin(), tr.split_index.end(), si);
    if (thr) std::copy(tr.threshold.begin(), tr.threshold.end(), thr);
    if (l) std::copy(tr.left.begin(), tr.left.end(), l);
    if (r) std::copy(tr.right.begin(), tr.right.end(), r);
    if (dl) std::copy(tr.default_left.begin(), tr.default_left.end(), dl);
    if (il) std::copy(tr.is_leaf.begin(), tr.is_leaf.end(), il);
    if (lv) std::copy(tr.leaf.begin(), tr.leaf.end(), lv);
    if (st) std::copy(tr.split_type.begin(), tr.split_type.end(), st);
    if (gain) std::copy(tr.gain.begin(), tr.gain.end(), gain);
    if (cover) std::copy(tr.cover.begin(), tr.cover.end(), cover);
    (void)nn;
}
void orc_tree_categories(const orc_model* m, uint32_t t, uint32_t* ss, uint32_t* sz, uint32_t* words) {
    const Tree& tr = m->trees[t];
    if (ss) std::copy(tr.seg_start.begin(), tr.seg_start.end(), ss);
    if (sz) std::copy(tr.seg_size.begin(), tr.seg_size.end(), sz);
    if (words) std::copy(tr.cat_words.begin(), tr.cat_words.end(), words);
}
void orc_tree_train_info(const orc_model* m, uint32_t t, uint32_t* sb, double* gs, double* hs) {
    const Tree& tr = m->trees[t];
    if (sb) std::copy(tr.split_bin.begin(), tr.split_bin.end(), sb);
    if (gs) std::copy(tr.grad_sum.begin(), tr.grad_sum.end(), gs);
    if (hs) std::copy(tr.hess_sum.begin(), tr.hess_sum.end(), hs);
}
void orc_tree_row_leaves(const orc_model* m, uint32_t t, uint32_t* out) {
    const Tree& tr = m->trees[t];
    std::copy(tr.row_leaf.begin(), tr.row_leaf.end(), out);
}
double orc_model_train_seconds(const orc_model* m) { return m->train_seconds; }
double orc_model_binning_seconds(const orc_model* m) { return m->binning_seconds; }
double orc_model_tree_seconds(const orc_model* m, uint32_t t) {
    return t < m->tree_seconds.size() ? m->tree_seconds[t] : 0.0;
}

int orc_predict(const orc_model* m, const float* x, uint64_t F, uint64_t n, int raw, float* out) {
    (void)F;
    predict_impl(m, x, n, false, F, raw != 0, 1, out);
    return 0;
}
int orc_predict_rows(const orc_model* m, const float* x, uint64_t F, uint64_t n, int raw, int omp,
                     float* out) {
    predict_impl(m, x, n, true, F, raw != 0, omp, out);
    return 0;
}

}  // extern "C"

// Known-answer and cross-language checks of the row sampler's generator.
extern "C" void orc_xoshiro256pp(const uint64_t state[4], uint32_t n, uint64_t* out) {
    OracleRowSampler r(0);
    for (int i = 0; i < 4; ++i) r.s[i] = state[i];
    for (uint32_t i = 0; i < n; ++i) out[i] = r.next();
}

extern "C" void orc_row_sample(uint64_t seed, uint64_t n, float rate, uint32_t draws, uint8_t* masks) {
    OracleRowSampler r(seed);
    std::vector<uint8_t> m;
    for (uint32_t d = 0; d < draws; ++d) {
        r.sample(n, rate, m);
        std::copy(m.begin(), m.end(), masks + (size_t)d * n);
    }
}
