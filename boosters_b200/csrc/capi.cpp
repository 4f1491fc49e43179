// capi.cpp — the extern "C" boundary (include/boosters_c.h).
// Every entry point catches engine errors and returns a status code; the
// message of the last failure is kept per thread.
#include <cmath>
#include <cstring>
#include <limits>
#include <string>

#include "../../include/boosters_c.h"
#include <cstdio>
#include <cstdlib>
#include "api_util.h"
#include "engine.h"
#include "nvtx_range.h"

struct bst_dataset {
    bst::HostDataset d;
};
struct bst_binned {
    bst::DeviceBinned b;
    int device = 0;
};
struct bst_model {
    std::unique_ptr<bst::Model> m;
};
struct bst_booster {
    std::unique_ptr<bst::Booster> b;
};
struct bst_server {
    bst::Server* s = nullptr;
    ~bst_server() { bst::server_destroy(s); }
};

namespace {

thread_local std::string g_err;

bst_status fail(bst_status code, const std::string& msg) {
    g_err = msg;
    return code;
}

template <class F>
bst_status guarded(F&& f) {
    try {
        g_err.clear();
        return f();
    } catch (const bst::Error& e) {
        return fail(e.code, e.msg);
    } catch (const std::bad_alloc&) {
        return fail(BST_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(BST_ERR_INVALID_ARGUMENT, e.what());
    }
}

// Checked build: a bounds-check violation recorded on `device` by the calls
// before this one turns a successful result into BST_ERR_CHECK.
bst_status check_after(int device, bst_status rc) {
#ifdef BST_CHECKED
    bst::CheckRecord r{};
    if (rc == BST_OK && bst::check_take(device, &r) && r.violations) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "bounds check failed %llu times; first at site %llu: index %llu, bound %llu",
                      r.violations, r.site, r.index, r.bound);
        return fail(BST_ERR_CHECK, msg);
    }
#else
    (void)device;
#endif
    return rc;
}

bool ratio_ok(float v) { return v > 0.0f && v <= 1.0f; }

template <class T>
void copy_out(T* dst, const std::vector<T>& src) {
    if (dst && !src.empty()) std::memcpy(dst, src.data(), sizeof(T) * src.size());
}

std::string fmt(float v) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%g", (double)v);
    return buf;
}

// GBDTConfig::validate (model/gbdt/config.rs:252-310) and engine limits.
bst_status check_config(const bst_config* c, bool for_training) {
    if (!c) return fail(BST_ERR_INVALID_ARGUMENT, "config is NULL");
    if (!(c->learning_rate > 0.0f)) return fail(BST_ERR_CONFIG, "learning_rate must be positive, got " + fmt(c->learning_rate));
    if (c->n_trees == 0) return fail(BST_ERR_CONFIG, "n_trees must be at least 1");
    const float* r[3] = {&c->subsample, &c->colsample_bytree, &c->colsample_bylevel};
    const char* rn[3] = {"subsample", "colsample_bytree", "colsample_bylevel"};
    for (int i = 0; i < 3; ++i)
        if (!ratio_ok(*r[i])) return fail(BST_ERR_CONFIG, std::string(rn[i]) + " must be in (0, 1], got " + fmt(*r[i]));
    const float* g[4] = {&c->lambda, &c->alpha, &c->min_child_weight, &c->min_gain};
    const char* gn[4] = {"lambda", "alpha", "min_child_weight", "min_gain"};
    for (int i = 0; i < 4; ++i)
        if (*g[i] < 0.0f) return fail(BST_ERR_CONFIG, std::string(gn[i]) + " must be non-negative, got " + fmt(*g[i]));
    // objective and sampling parameters (packages/boosters-python/src/objectives.rs
    // constructors, training/sampling/row.rs:64-75 RowSamplingParams::goss)
    if (c->objective == BST_OBJ_PINBALL || c->metric == BST_METRIC_QUANTILE) {
        if (c->n_quantiles == 0 || !c->quantile_alpha)
            return fail(BST_ERR_CONFIG, "pinball loss needs at least one quantile");
        for (uint32_t i = 0; i < c->n_quantiles; ++i)
            if (!(c->quantile_alpha[i] > 0.0f && c->quantile_alpha[i] < 1.0f))
                return fail(BST_ERR_CONFIG, "quantile alpha must be in (0, 1), got " + fmt(c->quantile_alpha[i]));
    }
    if ((c->objective == BST_OBJ_PSEUDO_HUBER || c->metric == BST_METRIC_HUBER) && !(c->huber_delta > 0.0f))
        return fail(BST_ERR_CONFIG, "huber_delta must be positive, got " + fmt(c->huber_delta));
    if (c->goss_top_rate != 0.0f || c->goss_other_rate != 0.0f) {
        if (!(c->goss_top_rate > 0.0f) || !(c->goss_other_rate > 0.0f))
            return fail(BST_ERR_CONFIG, "GOSS top_rate and other_rate must be positive");
        if (c->goss_top_rate + c->goss_other_rate > 1.0f)
            return fail(BST_ERR_CONFIG, "top_rate + other_rate must be <= 1.0");
        if (std::fabs(c->subsample - 1.0f) >= 1e-6f)
            return fail(BST_ERR_CONFIG, "GOSS and subsample < 1 cannot be combined");
    }
    if (!for_training) return BST_OK;
    if (c->objective < BST_OBJ_SQUARED || c->objective > BST_OBJ_HINGE)
        return fail(BST_ERR_UNSUPPORTED, "objective not supported by the GPU engine");
    if (c->objective == BST_OBJ_SOFTMAX && c->n_classes < 2) return fail(BST_ERR_CONFIG, "softmax needs n_classes >= 2");
    if (c->growth_strategy != BST_GROWTH_DEPTHWISE && c->growth_strategy != BST_GROWTH_LEAFWISE)
        return fail(BST_ERR_CONFIG, "unknown growth strategy");
    if (c->growth_strategy == BST_GROWTH_DEPTHWISE && c->max_depth > 24)
        return fail(BST_ERR_UNSUPPORTED, "max_depth > 24 is not supported by the GPU engine");
    if (c->growth_strategy == BST_GROWTH_LEAFWISE && c->max_leaves < 1)
        return fail(BST_ERR_CONFIG, "max_leaves must be at least 1");
    if (c->max_bins < 1) return fail(BST_ERR_CONFIG, "max_bins must be at least 1");
    if (c->precision != BST_PRECISION_FP32 && c->precision != BST_PRECISION_Q16 && c->precision != BST_PRECISION_Q8)
        return fail(BST_ERR_CONFIG, "unknown histogram precision " + std::to_string(c->precision));
    return BST_OK;
}

}  // namespace

namespace bst {
bst_status api_fail(bst_status code, const char* msg) { return fail(code, msg); }
bst_status api_check_config(const bst_config* c, bool for_training) { return check_config(c, for_training); }
void api_clear_error() { g_err.clear(); }
}  // namespace bst

extern "C" {

const char* bst_last_error(void) { return g_err.c_str(); }
const char* bst_version(void) { return "boosters-b200 0.1.0 (sm_100a)"; }
void bst_release_cached_memory(void) {
    bst::dev_cache_trim();
    bst::pinned_cache_trim();
}

void bst_config_default(bst_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->objective = BST_OBJ_SQUARED;
    c->n_classes = 0;
    c->metric = BST_METRIC_DEFAULT;
    c->n_trees = 100;
    c->learning_rate = 0.3f;
    c->growth_strategy = BST_GROWTH_DEPTHWISE;
    c->max_depth = 6;
    c->max_leaves = 31;
    c->max_onehot_cats = 4;
    c->lambda = 1.0f;
    c->alpha = 0.0f;
    c->min_child_weight = 1.0f;
    c->min_gain = 0.0f;
    c->min_samples_leaf = 1;
    c->subsample = 1.0f;
    c->colsample_bytree = 1.0f;
    c->colsample_bylevel = 1.0f;
    c->max_bins = 256;
    c->sparsity_threshold = 0.9f;
    c->enable_bundling = 1;
    c->max_categorical_cardinality = 0;
    c->binning_sample_cnt = 200000;
    c->early_stopping_rounds = -1;
    c->cache_size = 8;
    c->seed = 42;
    c->verbosity = 0;
    c->precision = BST_PRECISION_FP32;
    c->batched = 1;
    c->cuda_graph = 0;
    c->device = 0;
    c->record_leaves = 0;
    c->phase_timings = 0;
    c->autotune = 1;
    c->autotune_cache = nullptr;
    c->quantile_alpha = nullptr;
    c->n_quantiles = 0;
    c->huber_delta = 1.0f;
    c->goss_top_rate = 0.0f;
    c->goss_other_rate = 0.0f;
}

bst_status bst_config_validate(const bst_config* c) {
    g_err.clear();
    return check_config(c, false);
}

static bst_status dataset_create(const float* x, uint64_t F, uint64_t n, const float* y, uint32_t n_outputs,
                                 const float* w, const uint32_t* cat, uint32_t n_cat, bst_dataset** out, bool view) {
    return guarded([&]() -> bst_status {
        if (!out) return fail(BST_ERR_INVALID_ARGUMENT, "out is NULL");
        *out = nullptr;
        if (F == 0) return fail(BST_ERR_EMPTY_DATASET, "features cannot be empty");
        if (n > 0 && !x) return fail(BST_ERR_INVALID_ARGUMENT, "features is NULL");
        if (y && n_outputs == 0) return fail(BST_ERR_INVALID_ARGUMENT, "targets given with n_outputs == 0");
        for (uint32_t i = 0; i < n_cat; ++i)
            if (!cat || cat[i] >= F) return fail(BST_ERR_INVALID_ARGUMENT, "categorical feature index out of range");
        auto* ds = new bst_dataset();
        bst::HostDataset& d = ds->d;
        d.n = n;
        d.F = F;
        if (view)
            d.xv = x;
        else
            d.x.assign(x, x + F * n);
        if (y) {
            d.n_outputs = n_outputs;
            d.y.assign(y, y + (size_t)n_outputs * n);
        }
        if (w) {
            d.has_w = true;
            d.w.assign(w, w + n);
        }
        d.user_cat.assign(F, 0);
        for (uint32_t i = 0; i < n_cat; ++i) d.user_cat[cat[i]] = 1;
        *out = ds;
        return BST_OK;
    });
}

bst_status bst_dataset_create(const float* x, uint64_t F, uint64_t n, const float* y, uint32_t n_outputs,
                              const float* w, const uint32_t* cat, uint32_t n_cat, bst_dataset** out) {
    return dataset_create(x, F, n, y, n_outputs, w, cat, n_cat, out, false);
}

bst_status bst_dataset_create_view(const float* x, uint64_t F, uint64_t n, const float* y, uint32_t n_outputs,
                                   const float* w, const uint32_t* cat, uint32_t n_cat, bst_dataset** out) {
    return dataset_create(x, F, n, y, n_outputs, w, cat, n_cat, out, true);
}

void bst_dataset_free(bst_dataset* ds) { delete ds; }
uint64_t bst_dataset_n_samples(const bst_dataset* ds) { return ds ? ds->d.n : 0; }
uint64_t bst_dataset_n_features(const bst_dataset* ds) { return ds ? ds->d.F : 0; }

bst_status bst_binned_create(const bst_dataset* ds, const bst_config* cfg, bst_binned** out) {
    return guarded([&]() -> bst_status {
        if (!ds || !cfg || !out) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
        *out = nullptr;
        BST_CK(cudaSetDevice(cfg->device));
        auto* b = new bst_binned();
        b->device = cfg->device;
        cudaStream_t st;
        BST_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        try {
            bst::make_binned(ds->d, *cfg, st, b->b);
        } catch (...) {
            cudaStreamDestroy(st);
            delete b;
            throw;
        }
        cudaStreamDestroy(st);
        *out = b;
        return BST_OK;
    });
}

void bst_binned_free(bst_binned* b) { delete b; }
uint32_t bst_binned_n_columns(const bst_binned* b) { return b ? b->b.plan.n_cols() : 0; }

bst_status bst_binned_column_info(const bst_binned* b, uint32_t col, uint32_t* feature, uint32_t* n_bins,
                                  int32_t* is_cat, int32_t* has_missing, uint32_t* default_bin) {
    if (!b || col >= b->b.plan.n_cols()) return fail(BST_ERR_INVALID_ARGUMENT, "column out of range");
    const bst::BinPlan& p = b->b.plan;
    if (feature) *feature = p.col_feature[col];
    if (n_bins) *n_bins = p.col_nbins[col];
    if (is_cat) *is_cat = p.col_cat[col];
    if (has_missing) *has_missing = p.col_missing[col];
    if (default_bin) *default_bin = p.col_default[col];
    return BST_OK;
}

bst_status bst_binned_column_bounds(const bst_binned* b, uint32_t col, double* out) {
    if (!b || !out || col >= b->b.plan.n_cols()) return fail(BST_ERR_INVALID_ARGUMENT, "column out of range");
    const bst::Mapper& m = b->b.plan.mappers[b->b.plan.col_feature[col]];
    for (uint32_t i = 0; i < m.n_bins; ++i) out[i] = m.bin_to_value(i);
    return BST_OK;
}

bst_status bst_binned_column_bins(const bst_binned* b, uint32_t col, uint16_t* out) {
    return guarded([&]() -> bst_status {
        if (!b || !out || col >= b->b.plan.n_cols()) return fail(BST_ERR_INVALID_ARGUMENT, "column out of range");
        BST_CK(cudaSetDevice(b->device));
        const bst::BinPlan& p = b->b.plan;
        const uint64_t n = p.n;
        if (p.col_matrix[col] == 0) {
            std::vector<uint8_t> tmp(n);
            BST_CK(cudaMemcpy2D(tmp.data(), 1, b->b.bins8 + p.col_pos[col], p.s8, 1, n, cudaMemcpyDeviceToHost));
            for (uint64_t i = 0; i < n; ++i) out[i] = tmp[i];
        } else {
            BST_CK(cudaMemcpy2D(out, 2, b->b.bins16 + p.col_pos[col], (size_t)p.s16 * 2, 2, n, cudaMemcpyDeviceToHost));
        }
        return BST_OK;
    });
}

bst_status bst_gbdt_train(const bst_dataset* train, const bst_dataset* val, const bst_config* cfg,
                          uint32_t n_threads, bst_model** out) {
    return guarded([&]() -> bst_status {
        if (!out) return fail(BST_ERR_INVALID_ARGUMENT, "out is NULL");
        *out = nullptr;
        if (!train) return fail(BST_ERR_INVALID_ARGUMENT, "train dataset is NULL");
        bst_status rc = check_config(cfg, true);
        if (rc != BST_OK) return rc;
        if (train->d.n == 0) return fail(BST_ERR_EMPTY_DATASET, "dataset is empty");
        if (train->d.y.empty()) return fail(BST_ERR_MISSING_TARGETS, "dataset must have targets for training");
        // the validation set is read only by early stopping's evaluation
        // (trainer.rs:211-216: predictions only when a metric is set)
        const bool evaluates = cfg->early_stopping_rounds > 0 &&
                               bst::resolve_metric(cfg->metric, cfg->objective) != BST_METRIC_NONE && val;
        if (evaluates) {
            if (val->d.y.empty())  // eval.rs:242 ("validation set must have targets")
                return fail(BST_ERR_MISSING_TARGETS, "validation set must have targets");
            if (val->d.F < train->d.F)
                return fail(BST_ERR_INVALID_ARGUMENT, "validation set has fewer features than the training set");
        }
        BST_RANGE("bst.train");
        auto m = bst::train_model(train->d, *cfg, n_threads, evaluates ? &val->d : nullptr);
        rc = check_after(cfg->device, BST_OK);
        if (rc != BST_OK) return rc;
        *out = new bst_model{std::move(m)};
        return BST_OK;
    });
}

static bst_status predict_common(const bst_model* m, const bst_dataset* ds, bool raw, float* out) {
    return guarded([&]() -> bst_status {
        if (!m || !ds || !out) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
        if (ds->d.F < m->m->n_features)
            return fail(BST_ERR_INVALID_ARGUMENT, "dataset has fewer features than the model");
        bst::predict_host(*m->m, ds->d, raw, out);
        return BST_OK;
    });
}

bst_status bst_gbdt_predict(const bst_model* m, const bst_dataset* ds, uint32_t n_threads, float* out) {
    (void)n_threads;
    return predict_common(m, ds, false, out);
}
bst_status bst_gbdt_predict_raw(const bst_model* m, const bst_dataset* ds, uint32_t n_threads, float* out) {
    (void)n_threads;
    return predict_common(m, ds, true, out);
}

bst_status bst_gbdt_predict_device(const bst_model* m, const float* x, uint64_t n, uint64_t F, int32_t raw,
                                   float* out, void* stream) {
    return guarded([&]() -> bst_status {
        if (!m || (n && (!x || !out))) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
        if (F < m->m->n_features) return fail(BST_ERR_INVALID_ARGUMENT, "fewer features than the model");
        bst::predict_device(*m->m, x, n, F, raw != 0, out, (cudaStream_t)stream);
        return BST_OK;
    });
}

void bst_model_free(bst_model* m) { delete m; }

static bst_status copy_out(const void* src, size_t n, uint8_t** out, uint64_t* len) {
    uint8_t* b = static_cast<uint8_t*>(std::malloc(n ? n : 1));
    if (!b) return fail(BST_ERR_OUT_OF_MEMORY, "host allocation failed");
    if (n) std::memcpy(b, src, n);
    *out = b;
    *len = n;
    return BST_OK;
}

bst_status bst_model_to_json(const bst_model* model, int32_t pretty, uint8_t** out, uint64_t* len) {
    if (!model || !out || !len) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    return guarded([&]() -> bst_status {
        const std::string s = bst::model_to_json(*model->m, pretty != 0);
        return copy_out(s.data(), s.size(), out, len);
    });
}

bst_status bst_model_to_bstr_level(const bst_model* model, int32_t level, uint8_t** out, uint64_t* len) {
    if (!model || !out || !len) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    return guarded([&]() -> bst_status {
        const std::vector<uint8_t> b = bst::model_to_bstr(*model->m, level);
        return copy_out(b.data(), b.size(), out, len);
    });
}

bst_status bst_model_to_bstr(const bst_model* model, uint8_t** out, uint64_t* len) {
    return bst_model_to_bstr_level(model, BST_BSTR_DEFAULT_LEVEL, out, len);
}

bst_status bst_model_from_bytes(const uint8_t* data, uint64_t len, bst_model** out) {
    if (!out || (len && !data)) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    return guarded([&]() -> bst_status {
        std::unique_ptr<bst_model> h(new bst_model());
        h->m = bst::model_from_bytes(data, (size_t)len);
        *out = h.release();
        return BST_OK;
    });
}

void bst_buffer_free(void* p) { std::free(p); }

static bst_status write_file(const char* path, const void* data, size_t n) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(BST_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path + " for writing");
    const size_t w = n ? std::fwrite(data, 1, n, f) : 0;
    const int c = std::fclose(f);
    if (w != n || c != 0) return fail(BST_ERR_INVALID_ARGUMENT, std::string("write to ") + path + " failed");
    return BST_OK;
}

bst_status bst_model_write_json(const bst_model* model, const char* path, int32_t pretty) {
    if (!model || !path) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    return guarded([&]() -> bst_status {
        const std::string s = bst::model_to_json(*model->m, pretty != 0);
        return write_file(path, s.data(), s.size());
    });
}

bst_status bst_model_write_bstr_level(const bst_model* model, const char* path, int32_t level) {
    if (!model || !path) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    return guarded([&]() -> bst_status {
        const std::vector<uint8_t> b = bst::model_to_bstr(*model->m, level);
        return write_file(path, b.data(), b.size());
    });
}

bst_status bst_model_write_bstr(const bst_model* model, const char* path) {
    return bst_model_write_bstr_level(model, path, BST_BSTR_DEFAULT_LEVEL);
}

bst_status bst_model_load(const char* path, bst_model** out) {
    if (!path || !out) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    return guarded([&]() -> bst_status {
        FILE* f = std::fopen(path, "rb");
        if (!f) return fail(BST_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
        std::vector<uint8_t> buf;
        uint8_t chunk[1 << 16];
        size_t r;
        while ((r = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + r);
        std::fclose(f);
        std::unique_ptr<bst_model> h(new bst_model());
        h->m = bst::model_from_bytes(buf.data(), buf.size());
        *out = h.release();
        return BST_OK;
    });
}

uint32_t bst_crc32c(const uint8_t* data, uint64_t len) { return bst::crc32c_bytes(data, (size_t)len); }
uint32_t bst_model_n_trees(const bst_model* m) { return m ? (uint32_t)m->m->trees.size() : 0; }
uint32_t bst_model_n_groups(const bst_model* m) { return m ? m->m->n_groups : 0; }
uint32_t bst_model_n_features(const bst_model* m) { return m ? m->m->n_features : 0; }

bst_status bst_model_base_scores(const bst_model* m, float* out) {
    if (!m || !out) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memcpy(out, m->m->base.data(), sizeof(float) * m->m->base.size());
    return BST_OK;
}

bst_status bst_model_train_predictions(const bst_model* m, float* out) {
    if (!m || !out) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memcpy(out, m->m->train_pred.data(), sizeof(float) * m->m->train_pred.size());
    return BST_OK;
}

static const bst::HostTree* tree_at(const bst_model* m, uint32_t t) {
    if (!m || t >= m->m->trees.size()) {
        g_err = "tree index out of range";
        return nullptr;
    }
    return &m->m->trees[t];
}

bst_status bst_model_tree_info(const bst_model* m, uint32_t t, uint32_t* n_nodes, uint32_t* group,
                               uint32_t* n_words) {
    const bst::HostTree* tr = tree_at(m, t);
    if (!tr) return BST_ERR_INVALID_ARGUMENT;
    if (n_nodes) *n_nodes = (uint32_t)tr->split_index.size();
    if (group) *group = tr->group;
    if (n_words) *n_words = (uint32_t)tr->cat_words.size();
    return BST_OK;
}

bst_status bst_model_tree_nodes(const bst_model* m, uint32_t t, uint32_t* si, float* thr, uint32_t* l, uint32_t* r,
                                uint8_t* dl, uint8_t* il, float* lv, uint8_t* st, float* gain, float* cover) {
    const bst::HostTree* tr = tree_at(m, t);
    if (!tr) return BST_ERR_INVALID_ARGUMENT;
    copy_out(si, tr->split_index);
    copy_out(thr, tr->threshold);
    copy_out(l, tr->left);
    copy_out(r, tr->right);
    copy_out(dl, tr->default_left);
    copy_out(il, tr->is_leaf);
    copy_out(lv, tr->leaf);
    copy_out(st, tr->split_type);
    copy_out(gain, tr->gain);
    copy_out(cover, tr->cover);
    return BST_OK;
}

bst_status bst_model_tree_categories(const bst_model* m, uint32_t t, uint32_t* ss, uint32_t* sz, uint32_t* words) {
    const bst::HostTree* tr = tree_at(m, t);
    if (!tr) return BST_ERR_INVALID_ARGUMENT;
    copy_out(ss, tr->seg_start);
    copy_out(sz, tr->seg_size);
    copy_out(words, tr->cat_words);
    return BST_OK;
}

bst_status bst_model_tree_train_info(const bst_model* m, uint32_t t, uint32_t* sb, double* gs, double* hs) {
    const bst::HostTree* tr = tree_at(m, t);
    if (!tr) return BST_ERR_INVALID_ARGUMENT;
    copy_out(sb, tr->split_bin);
    copy_out(gs, tr->grad_sum);
    copy_out(hs, tr->hess_sum);
    return BST_OK;
}

bst_status bst_model_tree_row_leaves(const bst_model* m, uint32_t t, uint32_t* out) {
    const bst::HostTree* tr = tree_at(m, t);
    if (!tr) return BST_ERR_INVALID_ARGUMENT;
    if (tr->row_leaf.empty()) return fail(BST_ERR_INVALID_ARGUMENT, "model was trained without record_leaves");
    copy_out(out, tr->row_leaf);
    return BST_OK;
}

bst_status bst_model_train_timings(const bst_model* m, double* out8) {
    if (!m || !out8) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    for (int i = 0; i < 8; ++i) out8[i] = m->m->timings[i];
    return BST_OK;
}

bst_status bst_model_train_counters(const bst_model* m, uint64_t* out, uint32_t n) {
    if (!m || !out) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    const bst::Counters& c = m->m->counters;
    const uint64_t v[6] = {c.launches, c.hist_launches, c.hist_rows, c.hist_bytes, c.scan_launches, c.partition_rows};
    for (uint32_t i = 0; i < n && i < 6; ++i) out[i] = v[i];
    return BST_OK;
}

bst_status bst_model_tune_info(const bst_model* m, char* out, uint64_t cap, uint64_t* len) {
    if (!m || (cap && !out)) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    const std::string& s = m->m->tune_info;
    if (len) *len = s.size();
    if (cap) {
        const size_t k = std::min<size_t>(s.size(), (size_t)cap - 1);
        std::memcpy(out, s.data(), k);
        out[k] = '\0';
    }
    return BST_OK;
}

bst_status bst_booster_create(const bst_dataset* train, const bst_config* cfg, uint32_t n_threads,
                              bst_booster** out) {
    return guarded([&]() -> bst_status {
        if (!out || !train) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
        *out = nullptr;
        bst_status rc = check_config(cfg, true);
        if (rc != BST_OK) return rc;
        if (cfg->early_stopping_rounds > 0)
            return fail(BST_ERR_UNSUPPORTED, "early stopping needs bst_gbdt_train (the booster has no validation set)");
        if (train->d.n == 0) return fail(BST_ERR_EMPTY_DATASET, "dataset is empty");
        if (train->d.y.empty()) return fail(BST_ERR_MISSING_TARGETS, "dataset must have targets for training");
        *out = new bst_booster{std::make_unique<bst::Booster>(train->d, *cfg, n_threads)};
        return BST_OK;
    });
}

bst_status bst_booster_update(bst_booster* b, uint32_t n_rounds) {
    return guarded([&]() -> bst_status {
        if (!b) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
        b->b->update(n_rounds);
        return BST_OK;
    });
}

uint32_t bst_booster_n_rounds(const bst_booster* b) { return b ? b->b->rounds_done() : 0; }

bst_status bst_booster_model(const bst_booster* b, bst_model** out) {
    return guarded([&]() -> bst_status {
        if (!b || !out) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
        *out = new bst_model{b->b->snapshot()};
        return BST_OK;
    });
}

bst_status bst_booster_stats(const bst_booster* b, double* t8, uint64_t* c, uint32_t nc) {
    if (!b) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    const bst::Model& m = b->b->model();
    if (t8)
        for (int i = 0; i < 8; ++i) t8[i] = m.timings[i];
    if (c) {
        const bst::Counters& k = m.counters;
        const uint64_t v[6] = {k.launches, k.hist_launches, k.hist_rows, k.hist_bytes, k.scan_launches, k.partition_rows};
        for (uint32_t i = 0; i < nc && i < 6; ++i) c[i] = v[i];
    }
    return BST_OK;
}

void bst_booster_free(bst_booster* b) { delete b; }

bst_status bst_tree_grow(const bst_dataset* ds, const float* g, const float* h, const bst_config* cfg,
                         uint32_t n_threads, bst_model** out) {
    return guarded([&]() -> bst_status {
        if (!ds || !g || !h || !out) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
        *out = nullptr;
        bst_status rc = check_config(cfg, false);
        if (rc != BST_OK) return rc;
        if (cfg->growth_strategy != BST_GROWTH_DEPTHWISE && cfg->growth_strategy != BST_GROWTH_LEAFWISE)
            return fail(BST_ERR_CONFIG, "unknown growth strategy");
        if (ds->d.n == 0) return fail(BST_ERR_EMPTY_DATASET, "dataset is empty");
        auto m = bst::grow_one_tree(ds->d, g, h, *cfg, n_threads);
        *out = new bst_model{std::move(m)};
        return BST_OK;
    });
}

bst_status bst_model_create(uint32_t G, uint32_t F, int32_t objective, const float* base, bst_model** out) {
    return guarded([&]() -> bst_status {
        if (!out || G == 0 || !base) return fail(BST_ERR_INVALID_ARGUMENT, "bad argument");
        if (objective < BST_OBJ_SQUARED || objective > BST_OBJ_HINGE) return fail(BST_ERR_INVALID_ARGUMENT, "bad objective");
        auto m = std::make_unique<bst::Model>();
        m->n_groups = G;
        m->n_features = F;
        m->objective = objective;
        m->base.assign(base, base + G);
        int dev = 0;
        cudaGetDevice(&dev);
        cudaGetLastError();
        m->device = dev;
        *out = new bst_model{std::move(m)};
        return BST_OK;
    });
}

bst_status bst_model_add_tree(bst_model* mh, uint32_t group, uint32_t nn, const uint32_t* si, const float* thr,
                              const uint32_t* l, const uint32_t* r, const uint8_t* dl, const uint8_t* il,
                              const float* lv, const uint8_t* st, const uint32_t* ss, const uint32_t* sz,
                              const uint32_t* words, uint32_t n_words) {
    return guarded([&]() -> bst_status {
        if (!mh || nn == 0 || !si || !thr || !l || !r || !dl || !il || !lv)
            return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
        bst::Model& m = *mh->m;
        if (group >= m.n_groups) return fail(BST_ERR_INVALID_ARGUMENT, "group out of range");
        // validate: children in range and strictly after their parent (no cycles)
        for (uint32_t i = 0; i < nn; ++i) {
            if (il[i]) continue;
            if (l[i] >= nn || r[i] >= nn || l[i] <= i || r[i] <= i)
                return fail(BST_ERR_INVALID_ARGUMENT, "child index out of range or not after its parent");
            if (si[i] >= m.n_features) return fail(BST_ERR_INVALID_ARGUMENT, "split feature out of range");
            if (st && st[i] == 1 && ss && sz && (uint64_t)ss[i] + sz[i] > n_words)
                return fail(BST_ERR_INVALID_ARGUMENT, "category segment out of range");
        }
        bst::HostTree t;
        for (uint32_t i = 0; i < nn; ++i) t.alloc();
        for (uint32_t i = 0; i < nn; ++i) {
            t.split_index[i] = si[i];
            t.threshold[i] = thr[i];
            t.left[i] = l[i];
            t.right[i] = r[i];
            t.default_left[i] = dl[i] ? 1 : 0;
            t.is_leaf[i] = il[i] ? 1 : 0;
            t.leaf[i] = lv[i];
            t.split_type[i] = st ? st[i] : 0;
        }
        t.seg_start.assign(nn, 0);
        t.seg_size.assign(nn, 0);
        if (ss && sz) {
            t.seg_start.assign(ss, ss + nn);
            t.seg_size.assign(sz, sz + nn);
        }
        if (words && n_words) t.cat_words.assign(words, words + n_words);
        t.group = group;
        std::lock_guard<std::mutex> lk(m.mu);
        m.trees.push_back(std::move(t));
        m.dev.reset();  // rebuild the device forest on next use
        return BST_OK;
    });
}

// ---- component entry points ------------------------------------------------

bst_status bst_bin_values(const double* bounds, uint32_t n_bounds, int32_t missing, uint32_t default_bin,
                          int32_t is_cat, const int32_t* cats, uint32_t n_cats, const float* values,
                          uint64_t n, uint32_t* out) {
    return guarded([&]() -> bst_status {
        if ((n && (!values || !out)) || (is_cat && n_cats && !cats) || (!is_cat && n_bounds && !bounds))
            return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
        if (n == 0) return BST_OK;
        bst::Mapper m;
        m.categorical = is_cat != 0;
        m.missing = missing;
        m.default_bin = default_bin;
        if (m.categorical) {
            m.cats.assign(cats, cats + n_cats);
            m.n_bins = n_cats;
        } else {
            m.bounds.assign(bounds, bounds + n_bounds);
            m.n_bins = n_bounds;
        }
        const bool wide = m.n_bins > 256;
        bst::BinColumn bc;
        bc.matrix = wide ? 1 : 0;
        bc.pos = 0;
        bc.src = 0;
        bc.is_cat = m.categorical;
        bc.nan_bin = m.missing == bst::MISSING_NAN ? (m.n_bins ? m.n_bins - 1 : 0) : m.default_bin;
        bc.zero_bin = m.missing == bst::MISSING_ZERO ? m.default_bin : 0xFFFFFFFFu;
        std::vector<float> thr;
        std::vector<int32_t> cv;
        bc.off = 0;
        if (m.categorical) {
            std::vector<int32_t> sorted(m.cats);
            for (size_t i = 1; i < sorted.size(); ++i)
                if (sorted[i] <= sorted[i - 1]) return fail(BST_ERR_INVALID_ARGUMENT, "categories must be strictly increasing");
            cv = sorted;
            bc.n_cats = n_cats;
            bc.n_search = 0;
        } else {
            bc.n_cats = 0;
            bc.n_search = m.n_search();
            for (uint32_t j = 0; j < bc.n_search; ++j) thr.push_back(bst::f32_round_down(m.bounds[j]));
        }
        cudaStream_t st = nullptr;
        bst::DevArray<float> dx, dthr;
        bst::DevArray<int32_t> dc;
        bst::DevArray<bst::BinColumn> dcol;
        bst::DevArray<uint8_t> rec;
        dx.alloc(n);
        BST_CK(cudaMemcpy(dx.p, values, sizeof(float) * n, cudaMemcpyHostToDevice));
        dthr.alloc(std::max<size_t>(1, thr.size()));
        if (!thr.empty()) BST_CK(cudaMemcpy(dthr.p, thr.data(), sizeof(float) * thr.size(), cudaMemcpyHostToDevice));
        dc.alloc(std::max<size_t>(1, cv.size()));
        if (!cv.empty()) BST_CK(cudaMemcpy(dc.p, cv.data(), sizeof(int32_t) * cv.size(), cudaMemcpyHostToDevice));
        dcol.alloc(1);
        BST_CK(cudaMemcpy(dcol.p, &bc, sizeof(bc), cudaMemcpyHostToDevice));
        // one column: a 32-byte record per value, the bin at byte 0
        constexpr uint32_t REC = 32;
        rec.alloc(n * REC);
        bst::launch_bin_assign(dx.p, n, dcol.p, 1, dthr.p, dc.p, rec.p, REC, 0,
                               (uint32_t)std::max(thr.size(), cv.size()), st);
        BST_CK(cudaGetLastError());
        BST_CK(cudaDeviceSynchronize());
        if (!wide) {
            std::vector<uint8_t> t(n);
            BST_CK(cudaMemcpy2D(t.data(), 1, rec.p, REC, 1, n, cudaMemcpyDeviceToHost));
            for (uint64_t i = 0; i < n; ++i) out[i] = t[i];
        } else {
            std::vector<uint16_t> t(n);
            BST_CK(cudaMemcpy2D(t.data(), 2, rec.p, REC, 2, n, cudaMemcpyDeviceToHost));
            for (uint64_t i = 0; i < n; ++i) out[i] = t[i];
        }
        return BST_OK;
    });
}

// Power-of-two fixed-point scale with bound * 2^k < 2^62 (as k_fixed_scales).
static double fixed_scale(double bound) {
    if (!(bound > 0.0)) return 1.0;
    int e;
    std::frexp(bound, &e);
    int k = 62 - e;
    k = std::max(-1000, std::min(1000, k));
    return std::ldexp(1.0, k);
}

// The rule of k_fixed_scales: |q| <= 2^HIST_QBITS and n * 2^k * max < 2^62.
static double hist_scale(float m, uint64_t n) {
    if (!(m > 0.0f)) return 1.0;
    int e, en;
    std::frexp((double)m, &e);
    std::frexp((double)n, &en);
    int B = bst::HIST_QBITS;
    if (61 - en < B) B = 61 - en;
    int k = std::max(-1000, std::min(1000, B - e));
    return std::ldexp(1.0, k);
}

static bst::BinPlan plan_from_counts(const uint32_t* n_bins, uint32_t F, uint64_t n) {
    bst::BinPlan p;
    p.n = n;
    p.n_features = F;
    uint32_t off = 0;
    for (uint32_t f = 0; f < F; ++f) {
        p.col_feature.push_back(f);
        p.col_nbins.push_back(n_bins[f]);
        p.col_hist_off.push_back(off);
        p.col_default.push_back(0);
        p.col_cat.push_back(0);
        p.col_missing.push_back(0);
        if (n_bins[f] <= 256) {
            p.col_matrix.push_back(0);
            p.col_pos.push_back(p.f8++);
        } else {
            p.col_matrix.push_back(1);
            p.col_pos.push_back(p.f16++);
        }
        off += n_bins[f];
    }
    p.total_bins = off;
    p.s8 = (p.f8 + 15) / 16 * 16;
    p.s16 = (p.f16 + 7) / 8 * 8;
    return p;
}

bst_status bst_histogram_build(const uint16_t* bins, const uint32_t* n_bins, uint32_t F, uint64_t n,
                               const float* grad, const float* hess, const uint32_t* rows, uint64_t n_rows,
                               double* out) {
    return guarded([&]() -> bst_status {
        if (!bins || !n_bins || !grad || !hess || !out || F == 0) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
        if (n > 0xFFFFFFF0ull) return fail(BST_ERR_UNSUPPORTED, "too many rows");
        for (uint32_t f = 0; f < F; ++f)
            if (n_bins[f] == 0 || n_bins[f] > 4096) return fail(BST_ERR_UNSUPPORTED, "bins per feature must be in 1..4096");
        bst::BinPlan p = plan_from_counts(n_bins, F, n);
        const uint64_t cnt = rows ? n_rows : n;
        for (uint64_t i = 0; rows && i < n_rows; ++i)
            if (rows[i] >= n) return fail(BST_ERR_INVALID_ARGUMENT, "row index out of range");
        for (uint32_t f = 0; f < F; ++f)
            for (uint64_t i = 0; i < n; ++i)
                if (bins[(uint64_t)f * n + i] >= n_bins[f]) return fail(BST_ERR_INVALID_ARGUMENT, "bin out of range");
        std::vector<uint8_t> m8((size_t)n * p.s8, 0);
        std::vector<uint16_t> m16((size_t)n * p.s16, 0);
        for (uint32_t f = 0; f < F; ++f) {
            const uint16_t* src = bins + (uint64_t)f * n;
            if (p.col_matrix[f] == 0)
                for (uint64_t i = 0; i < n; ++i) m8[i * p.s8 + p.col_pos[f]] = (uint8_t)src[i];
            else
                for (uint64_t i = 0; i < n; ++i) m16[i * p.s16 + p.col_pos[f]] = src[i];
        }
        std::vector<float2> gh(n);
        float mg = 0.0f, mh = 0.0f;
        for (uint64_t i = 0; i < n; ++i) {
            gh[i] = make_float2(grad[i], hess[i]);
            if (std::fabs(grad[i]) <= 3.4e38f) mg = std::max(mg, std::fabs(grad[i]));
            if (std::fabs(hess[i]) <= 3.4e38f) mh = std::max(mh, std::fabs(hess[i]));
        }
        const double scale[4] = {hist_scale(mg, n), hist_scale(mh, n), 0, 0};
        std::vector<bst::HistTile> tiles;
        uint32_t max_smem = 0;
        bst::build_hist_tiles(p, tiles, max_smem);
        std::vector<bst::HistChunk> ch;
        for (uint64_t s = 0; s < cnt; s += 4096)
            ch.push_back(bst::HistChunk{0, (uint32_t)s, (uint32_t)std::min<uint64_t>(4096, cnt - s), rows ? 0u : 1u});
        bst::DevArray<uint8_t> d8;
        bst::DevArray<uint16_t> d16;
        bst::DevArray<float2> dgh;
        bst::DevArray<double> dsc;
        bst::DevArray<uint32_t> dr;
        bst::DevArray<bst::HistTile> dt;
        bst::DevArray<bst::HistChunk> dch;
        bst::DevArray<bst::HBin> dh;
        if (p.s8) {
            d8.alloc(m8.size());
            BST_CK(cudaMemcpy(d8.p, m8.data(), m8.size(), cudaMemcpyHostToDevice));
        }
        if (p.s16) {
            d16.alloc(m16.size());
            BST_CK(cudaMemcpy(d16.p, m16.data(), m16.size() * 2, cudaMemcpyHostToDevice));
        }
        dgh.alloc(std::max<uint64_t>(1, n));
        if (n) BST_CK(cudaMemcpy(dgh.p, gh.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
        dsc.alloc(4);
        BST_CK(cudaMemcpy(dsc.p, scale, sizeof(scale), cudaMemcpyHostToDevice));
        dr.alloc(std::max<uint64_t>(1, cnt));
        if (rows && cnt) BST_CK(cudaMemcpy(dr.p, rows, sizeof(uint32_t) * cnt, cudaMemcpyHostToDevice));
        dt.alloc(tiles.size());
        BST_CK(cudaMemcpy(dt.p, tiles.data(), sizeof(bst::HistTile) * tiles.size(), cudaMemcpyHostToDevice));
        dch.alloc(std::max<size_t>(1, ch.size()));
        if (!ch.empty()) BST_CK(cudaMemcpy(dch.p, ch.data(), sizeof(bst::HistChunk) * ch.size(), cudaMemcpyHostToDevice));
        dh.alloc(p.total_bins);
        BST_CK(cudaMemset(dh.p, 0, sizeof(bst::HBin) * p.total_bins));
        bst::GradRef gr{};
        gr.gh = dgh.p;
        gr.scale = dsc.p;
        gr.mode = bst::GRAD_F32;
        bst::launch_hist_build(dch.p, (uint32_t)ch.size(), dt.p, (uint32_t)tiles.size(), max_smem, dr.p, gr, d8.p,
                               p.s8, d16.p, p.s16, dh.p, p.total_bins, nullptr);
        BST_CK(cudaGetLastError());
        std::vector<bst::HBin> h(p.total_bins);
        BST_CK(cudaMemcpy(h.data(), dh.p, sizeof(bst::HBin) * p.total_bins, cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < p.total_bins; ++i) {
            out[2 * i] = (double)h[i].g / scale[0];
            out[2 * i + 1] = (double)h[i].h / scale[1];
        }
        return BST_OK;
    });
}

bst_status bst_find_split(const double* hist, const uint32_t* n_bins, const int32_t* is_cat, const int32_t* has_missing,
                          uint32_t F, double pg, double ph, uint32_t pc, const bst_config* cfg, uint32_t n_threads,
                          bst_split* out) {
    return guarded([&]() -> bst_status {
        if (!hist || !n_bins || !is_cat || !has_missing || !cfg || !out) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
        bst_status rc = check_config(cfg, false);
        if (rc != BST_OK) return rc;
        std::memset(out, 0, sizeof(*out));
        out->gain = -std::numeric_limits<float>::infinity();
        if (F == 0) return BST_OK;
        uint64_t total = 0;
        for (uint32_t f = 0; f < F; ++f) {
            if (is_cat[f] && n_bins[f] > 256) return fail(BST_ERR_UNSUPPORTED, "categorical features need <= 256 bins");
            total += n_bins[f];
        }
        // bound on every prefix sum: bins x max|bin| + |parent| (order-independent)
        double mg = 0.0, mh = 0.0;
        for (uint64_t i = 0; i < total; ++i) {
            mg = std::max(mg, std::fabs(hist[2 * i]));
            mh = std::max(mh, std::fabs(hist[2 * i + 1]));
        }
        const double sg = fixed_scale((double)total * mg + std::fabs(pg));
        const double sh = fixed_scale((double)total * mh + std::fabs(ph));
        std::vector<bst::HBin> h(total);
        for (uint64_t i = 0; i < total; ++i) {
            h[i].g = std::llrint(hist[2 * i] * sg);
            h[i].h = std::llrint(hist[2 * i + 1] * sh);
        }
        std::vector<bst::ScanColumn> cols(F);
        uint32_t off = 0;
        for (uint32_t f = 0; f < F; ++f) {
            cols[f] = bst::ScanColumn{n_bins[f], off, is_cat[f] ? 1u : 0u, has_missing[f] ? 1u : 0u};
            off += n_bins[f];
        }
        bst::ScanNode node{0, pc, 1u, 0u, std::llrint(pg * sg), std::llrint(ph * sh)};
        const double scale[4] = {sg, sh, 1.0 / sg, 1.0 / sh};
        bst::GainParamsDev gp;
        gp.lambda = (double)cfg->lambda;
        gp.min_gain = (double)cfg->min_gain;
        gp.min_child_weight = (double)cfg->min_child_weight;
        gp.min_samples_leaf = cfg->min_samples_leaf;
        gp.max_onehot_cats = cfg->max_onehot_cats;
        bst::DevArray<bst::HBin> dh;
        bst::DevArray<bst::ScanColumn> dc;
        bst::DevArray<bst::ScanNode> dn;
        bst::DevArray<double> ds;
        bst::DevArray<bst::ColCand> dcand;
        bst::DevArray<long long> dtot;
        bst::DevArray<bst::NodeSplit> dout;
        dh.alloc(total);
        BST_CK(cudaMemcpy(dh.p, h.data(), sizeof(bst::HBin) * total, cudaMemcpyHostToDevice));
        dc.alloc(F);
        BST_CK(cudaMemcpy(dc.p, cols.data(), sizeof(bst::ScanColumn) * F, cudaMemcpyHostToDevice));
        dn.alloc(1);
        BST_CK(cudaMemcpy(dn.p, &node, sizeof(node), cudaMemcpyHostToDevice));
        ds.alloc(4);
        BST_CK(cudaMemcpy(ds.p, scale, sizeof(scale), cudaMemcpyHostToDevice));
        dcand.alloc(F);
        dtot.alloc(2);
        dout.alloc(1);
        bst::launch_split_scan(dn.p, 1, dc.p, F, dh.p, total, ds.p, gp, dcand.p, dtot.p, nullptr);
        bst::launch_split_reduce(dcand.p, dtot.p, 1, F, (n_threads != 1 && F >= 16) ? 1 : 0, dout.p, nullptr);
        BST_CK(cudaGetLastError());
        bst::NodeSplit s;
        BST_CK(cudaMemcpy(&s, dout.p, sizeof(s), cudaMemcpyDeviceToHost));
        if (s.flags & 4u) {
            out->feature = s.col;
            out->gain = s.gain;
            out->default_left = (s.flags & 1u) ? 1 : 0;
            out->is_categorical = (s.flags & 2u) ? 1 : 0;
            out->bin = (s.flags & 2u) ? 0u : s.bin;  // SplitType::Categorical has no bin
            for (int q = 0; q < 4; ++q) out->left_cats[q] = s.cats[q];
        }
        return BST_OK;
    });
}

bst_status bst_quantize_gradients(const float* grad, const float* hess, uint64_t n, int32_t precision, uint64_t seed,
                                  uint32_t round, uint32_t output, int32_t* qg, int32_t* qh, double* steps) {
    if (!steps || (n && (!grad || !hess || !qg || !qh))) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    if (precision != BST_PRECISION_Q16 && precision != BST_PRECISION_Q8)
        return fail(BST_ERR_INVALID_ARGUMENT, "precision must be Q16 or Q8");
    if (n > 0xFFFFFFFFull) return fail(BST_ERR_INVALID_ARGUMENT, "at most 2^32 - 1 rows");
    return guarded([&]() -> bst_status {
        std::vector<float2> gh(n);
        for (uint64_t i = 0; i < n; ++i) gh[i] = make_float2(grad[i], hess[i]);
        bst::DevArray<float2> dgh;
        bst::DevArray<unsigned> dmax;
        bst::DevArray<double> dsteps;
        bst::DevArray<uint8_t> dq;
        const size_t qb = precision == BST_PRECISION_Q8 ? 2 : 4;
        dgh.alloc(std::max<uint64_t>(1, n));
        dmax.alloc(2);
        dsteps.alloc(4);
        dq.alloc(std::max<uint64_t>(1, n) * qb);
        if (n) BST_CK(cudaMemcpy(dgh.p, gh.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
        BST_CK(cudaMemset(dmax.p, 0, 2 * sizeof(unsigned)));
        bst::launch_maxabs(dgh.p, n, dmax.p, nullptr);
        bst::launch_quantize(precision, 1, dgh.p, n, dmax.p, seed, round, output, dq.p, dsteps.p, nullptr);
        BST_CK(cudaGetLastError());
        BST_CK(cudaMemcpy(steps, dsteps.p, 4 * sizeof(double), cudaMemcpyDeviceToHost));
        if (n == 0) return BST_OK;
        std::vector<uint8_t> hq(n * qb);
        BST_CK(cudaMemcpy(hq.data(), dq.p, n * qb, cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < n; ++i) {
            if (qb == 2) {
                qg[i] = (int8_t)hq[2 * i];
                qh[i] = (int8_t)hq[2 * i + 1];
            } else {
                int16_t a, b;
                std::memcpy(&a, &hq[4 * i], 2);
                std::memcpy(&b, &hq[4 * i + 2], 2);
                qg[i] = a;
                qh[i] = b;
            }
        }
        return BST_OK;
    });
}

bst_status bst_server_create(const bst_model* model, uint64_t mem_budget_bytes, uint64_t max_batch_rows,
                             int32_t raw, bst_server** out) {
    if (!model || !out) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    return guarded([&]() -> bst_status {
        std::unique_ptr<bst_server> h(new bst_server());
        h->s = bst::server_create(*model->m, mem_budget_bytes, max_batch_rows, raw != 0);
        *out = h.release();
        return BST_OK;
    });
}

bst_status bst_server_submit(bst_server* server, const float* rows, uint64_t n_rows, float* out, uint64_t* ticket) {
    if (!server || !ticket || (n_rows && (!rows || !out))) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    return guarded([&]() -> bst_status {
        *ticket = bst::server_submit(*server->s, rows, n_rows, out);
        return BST_OK;
    });
}

bst_status bst_server_wait(bst_server* server, uint64_t ticket, int64_t timeout_ms, uint64_t* submit_ns,
                           uint64_t* done_ns) {
    if (!server) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    return guarded([&]() -> bst_status {
        std::string err;
        const int st = bst::server_wait(*server->s, ticket, timeout_ms, submit_ns, done_ns, &err);
        return st == BST_OK ? BST_OK : fail((bst_status)st, err);
    });
}

bst_status bst_server_stats_get(bst_server* server, bst_server_stats* out) {
    if (!server || !out) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    bst::server_stats(*server->s, out);
    return BST_OK;
}

bst_status bst_server_trace(bst_server* server, bst_server_phase* out, uint64_t max, uint64_t* n) {
    if (!server || !n || (max && !out)) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    *n = bst::server_trace(*server->s, out, max);
    return BST_OK;
}

bst_status bst_server_replay(bst_server* server, const float* pool, uint64_t pool_rows, uint64_t n_req,
                             const uint64_t* arrival_ns, const uint64_t* row_off, const uint64_t* n_rows, float* out,
                             uint64_t ring, uint64_t ring_stride, uint64_t* latency_ns, uint64_t* span_ns) {
    if (!server || (n_req && (!pool || !arrival_ns || !row_off || !n_rows || !out || !latency_ns)))
        return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    return guarded([&]() -> bst_status {
        bst::server_replay(*server->s, pool, pool_rows, n_req, arrival_ns, row_off, n_rows, out, ring, ring_stride,
                           latency_ns, span_ns);
        return BST_OK;
    });
}

void bst_server_free(bst_server* server) { delete server; }

bst_status bst_metric_ex(int32_t metric, const float* p, uint32_t G, uint64_t n, const float* y, const float* w,
                         const float* alpha, uint32_t n_alpha, float delta, double* out) {
    if (!out || (n && (!p || !y))) return fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = 0.0;
    if (metric < BST_METRIC_RMSE || metric > BST_METRIC_MARGIN_ACCURACY)
        return fail(BST_ERR_INVALID_ARGUMENT, "unknown metric");
    if (metric == BST_METRIC_QUANTILE && (!alpha || n_alpha < G))
        return fail(BST_ERR_INVALID_ARGUMENT, "the quantile metric needs one alpha per output");
    if (metric == BST_METRIC_HUBER && !(delta > 0.0f)) return fail(BST_ERR_INVALID_ARGUMENT, "delta must be positive");
    bst::MetricParams mp;
    mp.alpha = alpha;
    mp.n_alpha = n_alpha;
    mp.delta = delta;
    *out = bst::metric_value(metric, p, G, n, y, w, mp);
    return BST_OK;
}

bst_status bst_metric(int32_t metric, const float* p, uint32_t G, uint64_t n, const float* y, const float* w,
                      double* out) {
    if (metric == BST_METRIC_QUANTILE) return fail(BST_ERR_INVALID_ARGUMENT, "the quantile metric needs bst_metric_ex");
    return bst_metric_ex(metric, p, G, n, y, w, nullptr, 0, 1.0f, out);
}

}  // extern "C"

bst_status bst_check_report(int32_t device, uint64_t* violations, uint32_t* site, uint64_t* index, uint64_t* bound) {
    return guarded([&]() -> bst_status {
#ifdef BST_CHECKED
        bst::CheckRecord r{};
        if (!bst::check_take(device, &r)) return fail(BST_ERR_CUDA, "cannot read the bounds-check record");
        if (violations) *violations = r.violations;
        if (site) *site = (uint32_t)r.site;
        if (index) *index = r.index;
        if (bound) *bound = r.bound;
        return BST_OK;
#else
        (void)device, (void)violations, (void)site, (void)index, (void)bound;
        return fail(BST_ERR_UNSUPPORTED, "not a checked build (libboosters_b200_checked.so has the bounds checks)");
#endif
    });
}
