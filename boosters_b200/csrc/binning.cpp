// binning.cpp — per-feature analysis, the row sample and the categorical
// mappers on the host; the numeric features' bounds come from a
// NumericBounds (the engine's device sort, mappers.cu).
//
// Semantics follow data/binned/feature_analysis.rs:313-569 (analysis and
// grouping) and data/binned/dataset.rs:592-750 (bin mappers). Features are
// processed in parallel; each feature's result depends only on its column.
#include "binning.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>
#include <unordered_set>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace bst {

namespace {

// `f64 as f32` with IEEE overflow to infinity.
float to_f32(double d) {
    const double lim = 0x1.ffffffp127;
    const double fmax = (double)std::numeric_limits<float>::max();
    if (d >= lim) return std::numeric_limits<float>::infinity();
    if (d <= -lim) return -std::numeric_limits<float>::infinity();
    if (d > fmax) return std::numeric_limits<float>::max();
    if (d < -fmax) return -std::numeric_limits<float>::max();
    return (float)d;
}

int32_t trunc_i32(double v) {  // `as i32`: truncate and saturate, NaN -> 0
    if (std::isnan(v)) return 0;
    if (v >= 2147483647.0) return 2147483647;
    if (v <= -2147483648.0) return (int32_t)(-2147483647 - 1);
    return (int32_t)v;
}

// Small open-addressing set of distinct f32 values (+0.0 and -0.0 are one
// value), tracking at most `limit` members like FeatureStats (feature_analysis.rs:296-346).
struct DistinctFloats {
    std::vector<uint32_t> slots;  // key bits + 1 (0 = empty)
    uint32_t mask = 0;
    size_t size = 0;
    float first = 0.0f;
    explicit DistinctFloats(size_t limit) {
        size_t cap = 16;
        while (cap < limit * 4) cap <<= 1;
        slots.assign(cap, 0);
        mask = (uint32_t)cap - 1;
    }
    static uint32_t key(float v) {
        if (v == 0.0f) v = 0.0f;
        uint32_t b;
        std::memcpy(&b, &v, 4);
        return b;
    }
    // returns true if v is new (and inserts it when `insert`)
    bool probe(float v, bool insert) {
        uint32_t k = key(v);
        uint32_t h = (k * 0x9E3779B1u) & mask;
        while (true) {
            uint32_t s = slots[h];
            if (s == 0) {
                if (insert) {
                    slots[h] = k + 1;
                    if (size == 0) first = v;
                    ++size;
                }
                return true;
            }
            if (s == k + 1) return false;
            h = (h + 1) & mask;
        }
    }
};

struct FeatureFacts {
    bool trivial = true, numeric = true, sparse = false, bundle_candidate = false;
    uint64_t n_nan = 0;
};

// v is a whole number: every float of magnitude 2^23 or more is; below
// that, exactly when truncation to int32 and back gives v (v - trunc(v) ==
// 0 for finite v; NaN and infinities are not whole).
inline bool whole(float v) {
    if (!(std::fabs(v) < 8388608.0f)) return std::isfinite(v);
    return (float)(int32_t)v == v;
}

FeatureFacts analyze(const float* col, uint64_t n, const bst_config& cfg, bool user_cat) {
    const size_t limit = std::max<size_t>(cfg.max_categorical_cardinality, cfg.max_bins) + 10;
    DistinctFloats uniq(limit);
    // three passes that each stop as early as their answer allows: the
    // NaN and nonzero counts (branch-free), the first non-whole value, the
    // distinct values until `limit` of them were seen
    uint64_t nan = 0, nonzero = 0;
#pragma omp simd reduction(+ : nan, nonzero)
    for (uint64_t i = 0; i < n; ++i) {
        const float v = col[i];
        nan += (v != v) ? 1u : 0u;
        nonzero += (v != 0.0f && v == v) ? 1u : 0u;
    }
    const uint64_t valid = n - nan;
    bool all_int = true;
    for (uint64_t i = 0; i < n && all_int; ++i) {
        const float v = col[i];
        if (v == v && !whole(v)) all_int = false;
    }
    bool exceeded = false;
    for (uint64_t i = 0; i < n && !exceeded; ++i) {
        const float v = col[i];
        if (v != v) continue;
        if (uniq.probe(v, false)) {
            if (uniq.size >= limit)
                exceeded = true;
            else
                uniq.probe(v, true);
        }
    }
    FeatureFacts f;
    const size_t n_unique = uniq.size;
    f.n_nan = nan;
    f.trivial = valid == 0 || (n_unique == 1 && uniq.first == 0.0f) || n_unique == 0;
    const bool binary = n_unique == 2;
    const bool auto_cat = !user_cat && all_int && n_unique <= cfg.max_categorical_cardinality;
    f.numeric = user_cat ? false : (binary ? true : !auto_cat);
    const float density = n == 0 ? 0.0f : (float)nonzero / (float)n;
    f.sparse = density <= (1.0f - cfg.sparsity_threshold);
    const double density64 = n == 0 ? 0.0 : (double)nonzero / (double)n;
    f.bundle_candidate = !f.numeric && density64 <= 1.0 - (double)cfg.sparsity_threshold;
    return f;
}

// dataset.rs:598-633: deterministic splitmix64 row sample used for bounds,
// in ascending row order (read off the bitmap of drawn rows).
std::vector<uint32_t> binning_sample(uint64_t n, uint64_t k) {
    std::vector<uint32_t> out;
    if (n <= k) return out;
    std::vector<uint64_t> seen((n + 63) / 64, 0);  // rows drawn so far
    uint64_t s = 0xD1B54A32D192ED03ULL ^ n, got = 0;
    while (got < k) {
        s += 0x9E3779B97F4A7C15ULL;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        const uint32_t r = (uint32_t)(z % n);
        uint64_t& word = seen[r >> 6];
        const uint64_t bit = 1ull << (r & 63u);
        if (!(word & bit)) {
            word |= bit;
            ++got;
        }
    }
    out.reserve(k);
    for (size_t wi = 0; wi < seen.size(); ++wi)
        for (uint64_t w = seen[wi]; w; w &= w - 1) out.push_back((uint32_t)(wi * 64 + (uint64_t)__builtin_ctzll(w)));
    return out;
}

}  // namespace

Mapper numeric_mapper_from_bounds(const double* bounds, uint32_t n_bounds, bool has_nan) {
    Mapper m;
    m.bounds.assign(bounds, bounds + n_bounds);
    m.n_bins = n_bounds;
    if (n_bounds > 1 && has_nan) {  // one finite value: a single bin and no NaN bin
        m.missing = MISSING_NAN;
        m.default_bin = n_bounds - 1;
    }
    return m;
}

float f32_round_down(double d) {
    float r = to_f32(d);
    if (std::isnan(d)) return r;
    if ((double)r > d) r = std::nextafter(r, -std::numeric_limits<float>::infinity());
    return r;
}

bst_status plan_binning(const float* x, uint64_t F, uint64_t n,
                        const std::vector<uint8_t>& user_cat, const bst_config& cfg,
                        NumericBounds& numeric, BinPlan& plan, std::string& err) {
    if (n == 0 || F == 0) {
        err = "dataset is empty";
        return BST_ERR_EMPTY_DATASET;
    }
    if (n > 0xFFFFFFF0ull) {
        err = "more than 2^32-16 rows are not supported";
        return BST_ERR_UNSUPPORTED;
    }
    plan = BinPlan();
    plan.n = n;
    plan.n_features = (uint32_t)F;
    plan.mappers.resize(F);
    plan.trivial.assign(F, 0);
    std::vector<FeatureFacts> facts(F);
    // the row sample (sequential draws) on one thread while the others
    // analyse the features
    std::vector<uint32_t> sample;
    std::thread sampler([&] { sample = binning_sample(n, cfg.binning_sample_cnt); });
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t f = 0; f < (int64_t)F; ++f) {
        const float* col = x + (uint64_t)f * n;
        const bool uc = (size_t)f < user_cat.size() && user_cat[f];
        facts[f] = analyze(col, n, cfg, uc);
    }
    sampler.join();

    // numeric features: bounds from the sampled values off the host, while
    // the host takes the categorical ones
    std::vector<uint32_t> num_f;
    std::vector<uint8_t> num_nan;
    for (uint64_t f = 0; f < F; ++f)
        if (!facts[f].trivial && facts[f].numeric) {
            num_f.push_back((uint32_t)f);
            num_nan.push_back(facts[f].n_nan > 0 ? 1 : 0);
        }
    if (!num_f.empty()) numeric.start(sample, num_f, num_nan, cfg.max_bins);

#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t f = 0; f < (int64_t)F; ++f) {
        const float* col = x + (uint64_t)f * n;
        const FeatureFacts& ff = facts[f];
        if (ff.trivial || ff.numeric) continue;
        {
            // every finite value's category, not a sample (dataset.rs:655-672):
            // categories in [0, 65536) in a bitmap, any others in a hash set;
            // the sorted distinct list is the same either way
            std::vector<uint64_t> small(1024, 0ull);
            std::unordered_set<int32_t> other;
            for (uint64_t i = 0; i < n; ++i) {
                const float v = col[i];
                if (!std::isfinite(v)) continue;
                const int32_t k = trunc_i32((double)v);
                if ((uint32_t)k < 65536u)
                    small[(uint32_t)k >> 6] |= 1ull << ((uint32_t)k & 63u);
                else
                    other.insert(k);
            }
            std::vector<int32_t> c(other.begin(), other.end());
            std::sort(c.begin(), c.end());  // negatives, then >= 65536
            const auto split = std::lower_bound(c.begin(), c.end(), 0);
            std::vector<int32_t> mid;
            for (uint32_t w = 0; w < 1024; ++w)
                for (uint64_t b = small[w]; b; b &= b - 1) mid.push_back((int32_t)(w * 64 + (uint32_t)__builtin_ctzll(b)));
            c.insert(split, mid.begin(), mid.end());
            if (c.empty()) c.push_back(0);
            Mapper m;
            m.categorical = true;
            m.n_bins = (uint32_t)c.size();
            m.cats = std::move(c);
            plan.mappers[f] = std::move(m);
        }
    }
    if (!num_f.empty()) numeric.finish(plan.mappers);

    for (uint64_t f = 0; f < F; ++f) {
        if (facts[f].trivial) {
            plan.trivial[f] = 1;
            continue;
        }
        // compute_groups (feature_analysis.rs:655-751) sends these to sparse
        // storage / EFB bundles, which the GPU engine does not implement.
        if (facts[f].sparse || (cfg.enable_bundling && facts[f].bundle_candidate)) {
            err = "feature " + std::to_string(f) +
                  " has density <= 1 - sparsity_threshold and would use sparse storage or a bundle, "
                  "which the GPU engine does not support; sparsity_threshold = 1 and enable_bundling = 0 "
                  "train it as a dense column";
            return BST_ERR_UNSUPPORTED;
        }
        const Mapper& m = plan.mappers[f];
        if (m.categorical && m.n_bins > 256) {
            err = "categorical feature " + std::to_string(f) + " has more than 256 categories";
            return BST_ERR_UNSUPPORTED;
        }
        if (m.n_bins > 4096) {
            err = "feature " + std::to_string(f) + " has more than 4096 bins";
            return BST_ERR_UNSUPPORTED;
        }
    }

    uint32_t off = 0;
    for (uint64_t f = 0; f < F; ++f) {
        if (plan.trivial[f]) continue;
        const Mapper& m = plan.mappers[f];
        plan.col_feature.push_back((uint32_t)f);
        plan.col_nbins.push_back(m.n_bins);
        plan.col_hist_off.push_back(off);
        plan.col_default.push_back(m.default_bin);
        plan.col_cat.push_back(m.categorical ? 1 : 0);
        plan.col_missing.push_back(m.missing != MISSING_NONE ? 1 : 0);
        if (m.n_bins <= 256) {
            plan.col_matrix.push_back(0);
            plan.col_pos.push_back(plan.f8++);
        } else {
            plan.col_matrix.push_back(1);
            plan.col_pos.push_back(plan.f16++);
        }
        off += m.n_bins;
    }
    plan.total_bins = off;
    // One record per row: the u8 columns, then from a 16-byte boundary the
    // u16 columns, the whole padded to a 32-byte sector (80 u8 + 20 u16
    // columns: 128 bytes, one cache line). Rows start on sector boundaries,
    // so every aligned 16- or 32-byte window of a row lies in one sector and
    // a gathered row costs exactly its sectors.
    plan.u16_off = plan.f16 ? (plan.f8 + 15) / 16 * 16 : plan.f8;
    plan.rec = (plan.u16_off + 2 * plan.f16 + 31) / 32 * 32;
    plan.s8 = plan.rec;       // row stride of the u8 view, bytes
    plan.s16 = plan.rec / 2;  // row stride of the u16 view (record + u16_off), elements
    return BST_OK;
}

}  // namespace bst
